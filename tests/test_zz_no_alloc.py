"""The entry point that allocates nothing (bls_reduce_schur_dense_noalloc), against the plan-based reduction.

Callers whose device memory belongs to an allocator they do not own (CUDA.jl's pool, PyTorch's caching allocator) or
who are held to a fixed budget cannot let the library call cudaMalloc; for them bls_reduce_schur_dense_noalloc takes
the structure's index arrays from the caller and keeps its scratch in a static device array. This test calls it
through the C ABI twice in a row on the dense 50 x 2,000 scene and compares S and g_S with bls_reduce_schur_dense
within the tolerances of the other device tests (1e-12 relative in FP64, 1e-5 in FP32 against the FP32 plan path),
and checks that sizes beyond its limit are refused without any work. This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def relerr(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def problem(bls):
    p = bls.scenes.hessian_problem(bls.scenes.workload("dense_50x2000"), dense=True)
    st = p.structure
    assert np.array_equal(st.coffsets, 18 * np.arange(len(st.coffsets)))   # the canonical layout the call requires
    assert np.array_equal(st.eoffsets, 9 * np.arange(st.neblocks))
    return p


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_noalloc_matches_plan_twice(bls, problem, dtype, tol):
    p = problem
    st = p.structure
    nr = st.nr
    t = lambda a, d=dtype: torch.from_numpy(np.ascontiguousarray(a)).to(device=DEV, dtype=d)
    E, Cd, R = t(p.E), t(p.C), t(p.R)
    b_r, b_e = t(p.b_r, torch.float64), t(p.b_e, torch.float64)
    sr, se = t(p.scaling_r, torch.float64), t(p.scaling_e, torch.float64)
    eptr = t(st.eliminated_ptr, torch.int64)
    eret = t(st.entry_retained, torch.int64)
    # the reset system and the plan path's result
    ws = bls.SchurReductionWorkspace(st)
    S0 = torch.zeros(nr * nr, dtype=dtype, device=DEV)
    bls.reset_schur_dense(S0, R, sr, p.lam, ws)
    S_ref = S0.clone()
    g_ref = torch.zeros(nr, dtype=torch.float64, device=DEV)
    assert bls.reduce_schur_dense(S_ref, g_ref, b_r, b_e, se, p.lam, st, E, Cd, ws)
    L = bls._lib.gpu()
    code = bls._lib.BLS_F64 if dtype == torch.float64 else bls._lib.BLS_F32
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        S = S0.clone()
        g = torch.full((nr,), 99.0, dtype=torch.float64, device=DEV)
        fb = C.c_int64(-1)
        rc = L.bls_reduce_schur_dense_noalloc(stream, code, st.nrblocks, st.neblocks, len(st.entry_retained),
                                              C.c_void_p(eptr.data_ptr()), C.c_void_p(eret.data_ptr()), C.c_void_p(S.data_ptr()),
                                              C.c_void_p(g.data_ptr()), C.c_void_p(b_r.data_ptr()), C.c_void_p(b_e.data_ptr()),
                                              C.c_void_p(se.data_ptr()), p.lam, C.c_void_p(E.data_ptr()), C.c_void_p(Cd.data_ptr()),
                                              C.byref(fb))
        assert rc == 0 and fb.value == 0, (call, rc, L.bls_last_error())
        Su = np.triu(S.double().cpu().numpy().reshape(nr, nr, order="F"))
        Sr = np.triu(S_ref.double().cpu().numpy().reshape(nr, nr, order="F"))
        assert relerr(Su, Sr) < tol, call
        assert relerr(g.cpu().numpy(), g_ref.cpu().numpy()) < max(tol, 1e-12), call


def test_noalloc_reports_failure_and_refuses_oversize(bls, problem):
    p = problem
    st = p.structure
    nr = st.nr
    t = lambda a, d=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to(device=DEV, dtype=d)
    E = p.E.copy()
    v = np.array([1.0, 2.0, 3.0])
    for e in (4, 9):                       # two singular points (undamped): the lowest is reported, 1-based
        E[9 * e:9 * e + 9] = np.outer(v, v).ravel(order="F")
    L = bls._lib.gpu()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [t(st.eliminated_ptr, torch.int64), t(st.entry_retained, torch.int64)]
    S = torch.full((nr * nr,), 3.0, dtype=torch.float64, device=DEV)
    g = torch.full((nr,), 5.0, dtype=torch.float64, device=DEV)
    b_r, b_e, se, Et, Ct = t(p.b_r), t(p.b_e), t(np.zeros_like(p.scaling_e)), t(E), t(p.C)
    ptrs = lambda *ts: [C.c_void_p(x.data_ptr()) for x in ts]
    fb = C.c_int64(-1)
    rc = L.bls_reduce_schur_dense_noalloc(stream, bls._lib.BLS_F64, st.nrblocks, st.neblocks, len(st.entry_retained), *ptrs(*args, S, g, b_r, b_e, se),
                                          0.0, *ptrs(Et, Ct), C.byref(fb))
    assert rc == bls._lib.BLS_NOT_PD and fb.value == 5
    assert torch.all(S == 3.0) and torch.all(g == 5.0)     # untouched, as the reference returns before phase 2
    rc = L.bls_reduce_schur_dense_noalloc(stream, bls._lib.BLS_F64, st.nrblocks, 65537, len(st.entry_retained), *ptrs(*args, S, g, b_r, b_e, se),
                                          0.0, *ptrs(Et, Ct), C.byref(fb))
    assert rc == bls._lib.BLS_EUNSUPPORTED and b"65536" in L.bls_last_error()


def _noalloc_args(bls, p, E=None, scaling_e=None, eret=None):
    st = p.structure
    nr = st.nr
    t = lambda a, d=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to(device=DEV, dtype=d)
    bufs = dict(eptr=t(st.eliminated_ptr, torch.int64), eret=t(st.entry_retained if eret is None else eret, torch.int64),
                S=torch.full((nr * nr,), 3.0, dtype=torch.float64, device=DEV), g=torch.full((nr,), 5.0, dtype=torch.float64, device=DEV),
                b_r=t(p.b_r), b_e=t(p.b_e), se=t(p.scaling_e if scaling_e is None else scaling_e), E=t(p.E if E is None else E),
                C=t(p.C))
    return bufs


def _call(bls, p, b, failed_block):
    st = p.structure
    L = bls._lib.gpu()
    v = lambda x: C.c_void_p(x.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return L.bls_reduce_schur_dense_noalloc(stream, bls._lib.BLS_F64, st.nrblocks, st.neblocks, len(st.entry_retained), v(b["eptr"]),
                                           v(b["eret"]), v(b["S"]), v(b["g"]), v(b["b_r"]), v(b["b_e"]), v(b["se"]), p.lam, v(b["E"]),
                                           v(b["C"]), failed_block)


def test_noalloc_async_verdict_is_queried(bls, problem):
    """With failed_block NULL the call queues its work and keeps its verdict in the static array's status words;
    bls_reduce_schur_dense_noalloc_status reads it (the lowest failing block, 1-based), and a clean call reads OK."""
    p = problem
    L = bls._lib.gpu()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    E = p.E.copy()
    v = np.array([1.0, 2.0, 3.0])
    for e in (7, 11):
        E[9 * e:9 * e + 9] = np.outer(v, v).ravel(order="F")
    b = _noalloc_args(bls, p, E=E, scaling_e=np.zeros_like(p.scaling_e))
    assert _call(bls, p, b, None) == 0
    fb = C.c_int64(-1)
    assert L.bls_reduce_schur_dense_noalloc_status(stream, C.byref(fb)) == bls._lib.BLS_NOT_PD and fb.value == 8
    assert torch.all(b["S"] == 3.0) and torch.all(b["g"] == 5.0)
    b = _noalloc_args(bls, p)
    assert _call(bls, p, b, None) == 0
    fb = C.c_int64(-1)
    assert L.bls_reduce_schur_dense_noalloc_status(stream, C.byref(fb)) == 0 and fb.value == 0
    assert not torch.all(b["S"] == 3.0)


@pytest.mark.parametrize("case", ["descending", "out_of_range", "negative_scaling", "nan_scaling"])
def test_noalloc_rejects_bad_arguments_untouched(bls, problem, case):
    """A malformed structure (entry_retained not ascending within a point, or beyond nrblocks) and a negative or NaN
    scaling_e entry are BLS_EINVAL, found by the call's own checks before its atomics touch S or g_S: both stay as
    they were, synchronously and through the status query."""
    p = problem
    st = p.structure
    L = bls._lib.gpu()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    eret, se = None, None
    e = 3
    a, z = int(st.eliminated_ptr[e]), int(st.eliminated_ptr[e + 1])
    assert z - a >= 2
    if case == "descending":
        eret = st.entry_retained.copy()
        eret[a], eret[a + 1] = eret[a + 1], eret[a]
    elif case == "out_of_range":
        eret = st.entry_retained.copy()
        eret[z - 1] = st.nrblocks
    elif case == "negative_scaling":
        se = p.scaling_e.copy()
        se[10] = -1.0
    else:
        se = p.scaling_e.copy()
        se[10] = np.nan
    for sync in (True, False):
        b = _noalloc_args(bls, p, scaling_e=se, eret=eret)
        fb = C.c_int64(-1)
        if sync:
            rc = _call(bls, p, b, C.byref(fb))
        else:
            assert _call(bls, p, b, None) == 0
            rc = L.bls_reduce_schur_dense_noalloc_status(stream, C.byref(fb))
        assert rc == bls._lib.BLS_EINVAL, (case, sync, rc)
        msg = L.bls_last_error()
        assert (b"scaling_e" in msg) if "scaling" in case else (b"malformed structure" in msg and b"block 4 " in msg), msg
        torch.cuda.synchronize()
        assert torch.all(b["S"] == 3.0) and torch.all(b["g"] == 5.0), (case, sync)
