"""Device Schur reduction through the C ABI against the oracle (the reference's algorithm restated on the CPU).

FP64: S, g_S and the back-substituted x_e within 1e-12 relative of the oracle (test/schur.jl:223-237 bounds the
reference's own solutions at 1e-12; the device sums in another order, as the reference's threaded path does, which
test/schur.jl:399-400 bounds at 1e-13). Mixed form (FP32 storage and accumulation, FP64 inverse): against the FP64
oracle on the same FP32 inputs, within 1e-4 relative in S (FP32 accumulation of ~k^2 terms of size |C|^2/|E|).
Failure reporting (lowest failing block, outputs untouched), argument checks, dense and sparse, conditioning scales.
"""
import numpy as np
import pytest
import torch

import oracle as orc
from fixtures import COUPLED_GROUPS, GAUGE, MIXED_DIMS, SCHUR_JL, STANDARD, make_problem, split_hessian

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


def run_both(bls, st, ost, pat, opat, E, Cd, R, b_r, b_e, sc_r, sc_e, lam, dense, dtype, s_r=None, s_e=None, kernel="pairs",
             stage_unit=None):
    """One reset + reduce + back-substitution on the device and in the oracle (FP64, on the same stored values)."""
    npdt = np.float32 if dtype == torch.float32 else np.float64
    E32, C32, R32 = E.astype(npdt), Cd.astype(npdt), R.astype(npdt)
    nr = st.nr
    ws = bls.SchurReductionWorkspace(st, pat)
    ws.set_kernel(kernel)
    if stage_unit is not None:
        ws.set_stage_unit(stage_unit)
    g = torch.zeros(nr, dtype=torch.float64, device=DEV)
    args = dict(s_r=None if s_r is None else cu(s_r), s_e=None if s_e is None else cu(s_e))
    if dense:
        S = torch.zeros(nr * nr, dtype=dtype, device=DEV)
        bls.reset_schur_dense(S, cu(R32), cu(sc_r), lam, ws, s_r=args["s_r"])
        ok = bls.reduce_schur_dense(S, g, cu(b_r), cu(b_e), cu(sc_e), lam, st, cu(E32), cu(C32), ws, **args)
    else:
        S = torch.zeros(pat.nnz, dtype=dtype, device=DEV)
        bls.reset_schur_sparse(S, cu(R32), None, None, cu(sc_r), lam, ws, s_r=args["s_r"])
        ok = bls.reduce_schur_sparse(S, g, cu(b_r), cu(b_e), cu(sc_e), lam, st, cu(E32), cu(C32), None, None, None, None, ws, **args)
    # oracle in FP64 on the stored (possibly FP32-rounded) values
    work = orc.Work(ost, 1)
    og = np.zeros(nr)
    if dense:
        oS = np.zeros(nr * nr)
        orc.reset_schur_dense(ost, oS, R32.astype(np.float64), sc_r, lam, s_r)
        ook, ofb = orc.reduce_schur_dense(ost, work, oS, og, b_r, b_e, sc_e, lam, E32.astype(np.float64), C32.astype(np.float64), s_r, s_e)
    else:
        oS = np.zeros(opat.nnz)
        orc.reset_schur_sparse(ost, opat, oS, R32.astype(np.float64), sc_r, lam, s_r)
        ook, ofb = orc.reduce_schur_sparse(ost, opat, work, oS, og, b_r, b_e, sc_e, lam, E32.astype(np.float64), C32.astype(np.float64), s_r, s_e)
    out = dict(ok=ok, fb=ws.failed_block, ook=ook, ofb=ofb, S=S.double().cpu().numpy(), oS=oS, g=g.cpu().numpy(), og=og, ws=ws, work=work)
    if ok and ook:
        x_r = np.random.default_rng(0).standard_normal(nr)
        x_e = torch.zeros(st.ne, dtype=torch.float64, device=DEV)
        bls.backsubstitute(x_e, cu(x_r), st, cu(C32), ws, s_r=args["s_r"], s_e=args["s_e"])
        ox_e = np.zeros(st.ne)
        orc.backsubstitute(ost, work, ox_e, x_r, C32.astype(np.float64), s_r, s_e)
        out.update(x_e=x_e.cpu().numpy(), ox_e=ox_e)
    return out


def fixture_system(bls, fx, seed=7, lam=0.5):
    rng = np.random.default_rng(seed)
    rr = fx.get("rr_pairs", [])
    H, b = make_problem(rng, fx["r_dims"], fx["e_dims"], fx["couplings"], rr)
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    return H, b, st, ost, rr, 1.0 + rng.random(len(b))


@pytest.mark.parametrize("name", ["schur_jl", "standard", "coupled_groups", "gauge", "mixed_dims"])
@pytest.mark.parametrize("dense", [False, True])
def test_fixture_fp64(bls, name, dense):
    fx = {"schur_jl": SCHUR_JL, "standard": STANDARD, "coupled_groups": COUPLED_GROUPS, "gauge": GAUGE, "mixed_dims": MIXED_DIMS}[name]
    H, b, st, ost, rr, sc = fixture_system(bls, fx)
    pat = None if dense else bls.build_schur_pattern(st, rr)
    opat = None if dense else orc.Pattern(ost, rr)
    E, Cd, R = split_hessian(H, st, pat)
    nr = st.nr
    o = run_both(bls, st, ost, pat, opat, E, Cd, R, b[:nr], b[nr:], sc[:nr], sc[nr:], 0.5, dense, torch.float64)
    assert o["ok"] and o["ook"]
    assert relerr(o["S"], o["oS"]) < 1e-12
    assert relerr(o["g"], o["og"]) < 1e-12
    assert relerr(o["x_e"], o["ox_e"]) < 1e-12


@pytest.mark.parametrize("dense", [False, True])
def test_fixture_conditioned_scales(bls, dense):
    """Power-of-two conditioning scales applied at read (src/conditioning.jl:99-150)."""
    H, b, st, ost, rr, sc = fixture_system(bls, STANDARD, seed=11)
    pat = None if dense else bls.build_schur_pattern(st, rr)
    opat = None if dense else orc.Pattern(ost, rr)
    E, Cd, R = split_hessian(H, st, pat)
    rng = np.random.default_rng(2)
    s = np.ldexp(1.0, rng.integers(-6, 7, len(b)))
    nr = st.nr
    o = run_both(bls, st, ost, pat, opat, E, Cd, R, b[:nr], b[nr:], sc[:nr], sc[nr:], 0.3, dense, torch.float64, s_r=s[:nr], s_e=s[nr:])
    assert o["ok"] and o["ook"]
    assert relerr(o["S"], o["oS"]) < 1e-12 and relerr(o["g"], o["og"]) < 1e-12 and relerr(o["x_e"], o["ox_e"]) < 1e-12


@pytest.mark.parametrize("dense", [False, True])
def test_rank_one_block_reports_lowest(bls, dense):
    H, b, st, ost, rr, sc = fixture_system(bls, SCHUR_JL, seed=5)
    nr = st.nr
    v = np.random.default_rng(9).standard_normal(3)
    H[nr:nr + 3, nr:nr + 3] = np.outer(v, v)
    H[nr + 12:nr + 15, nr + 12:nr + 15] = np.outer(v, v)   # a second, higher failing block
    pat = None if dense else bls.build_schur_pattern(st)
    opat = None if dense else orc.Pattern(ost)
    E, Cd, R = split_hessian(H, st, pat)
    o = run_both(bls, st, ost, pat, opat, E, Cd, R, b[:nr], b[nr:], sc[:nr], np.ones(st.ne), 0.0, dense, torch.float64)
    assert not o["ok"] and not o["ook"]
    assert o["fb"] == o["ofb"] == 1
    # S is left as the reset wrote it, g_S untouched (the reference returns before phase 2)
    assert relerr(o["S"], o["oS"]) < 1e-15
    assert np.all(o["g"] == 0.0)


def test_bad_damping_is_rejected_without_writes(bls):
    H, b, st, ost, rr, sc = fixture_system(bls, STANDARD)
    pat = bls.build_schur_pattern(st)
    E, Cd, R = split_hessian(H, st, pat)
    nr = st.nr
    ws = bls.SchurReductionWorkspace(st, pat)
    S = torch.full((pat.nnz,), 7.0, dtype=torch.float64, device=DEV)
    g = torch.full((nr,), 5.0, dtype=torch.float64, device=DEV)
    with pytest.raises(bls.ArgumentError):
        bls.reset_schur_sparse(S, cu(R), None, None, cu(sc[:nr]), -1.0, ws)
    bad = sc[:nr].copy()
    bad[3] = np.nan
    bls.reset_schur_sparse(S, cu(R), None, None, cu(bad), 0.1, ws)   # recorded, reported by the next reduction
    assert torch.all(S == 7.0)
    with pytest.raises(bls.ArgumentError, match="scaling_r must be finite and non-negative, but entry 4"):
        bls.reduce_schur_sparse(S, g, cu(b[:nr]), cu(b[nr:]), cu(sc[nr:]), 0.1, st, cu(E), cu(Cd), None, None, None, None, ws)
    assert torch.all(S == 7.0) and torch.all(g == 5.0)
    bls.reset_schur_sparse(S, cu(R), None, None, cu(sc[:nr]), 0.1, ws)
    bad_e = sc[nr:].copy()
    bad_e[0] = -1.0
    S2 = S.clone()
    with pytest.raises(bls.ArgumentError, match="scaling_e"):
        bls.reduce_schur_sparse(S, g, cu(b[:nr]), cu(b[nr:]), cu(bad_e), 0.1, st, cu(E), cu(Cd), None, None, None, None, ws)
    assert torch.equal(S, S2) and torch.all(g == 5.0)
    with pytest.raises(bls.ArgumentError):
        bls.reduce_schur_sparse(S, g, cu(b[:nr]), cu(b[nr:]), cu(sc[nr:]), float("inf"), st, cu(E), cu(Cd), None, None, None, None, ws)


def scene_system(bls, name, ncams, npoints, dense=False, seed=None):
    spec = bls.scenes.scaled_down(bls.scenes.workload(name), ncams, npoints, seed)
    p = bls.scenes.hessian_problem(spec, dense=dense)
    st = p.structure
    bs, el, ptr, idx = bls.scenes.Scene(spec).description()
    ost = orc.Structure.from_description(bs, (ptr, idx), el)
    opat = None if dense else orc.Pattern(ost)
    return p, st, ost, opat


@pytest.mark.parametrize("kernel", ["stage", "columns", "pairs", "lanes", "tiles", "points"])
@pytest.mark.parametrize("name,ncams,npoints,dense", [
    ("dense_50x2000", 50, 2000, True),            # the dense workload at full size
    ("sparse_1000x200k", 120, 8000, False),
    ("batched_256", 60, 3000, False),
    ("pcg_10000x1M", 150, 6000, False),
])
def test_scene_fp64_matches_oracle(bls, name, ncams, npoints, dense, kernel):
    p, st, ost, opat = scene_system(bls, name, ncams, npoints, dense)
    o = run_both(bls, st, ost, p.pattern, opat, p.E, p.C, p.R, p.b_r, p.b_e, p.scaling_r, p.scaling_e, p.lam, dense, torch.float64,
                 kernel=kernel)
    assert o["ok"] and o["ook"]
    assert relerr(o["S"], o["oS"]) < 1e-12
    assert relerr(o["g"], o["og"]) < 1e-12
    assert relerr(o["x_e"], o["ox_e"]) < 1e-10


@pytest.mark.parametrize("kernel", ["stage", "columns", "pairs", "lanes", "tiles", "points"])
@pytest.mark.parametrize("name,ncams,npoints", [("sparse_1000x200k", 120, 8000), ("pcg_10000x1M", 150, 6000)])
def test_scene_mixed_matches_fp64_oracle(bls, name, ncams, npoints, kernel):
    p, st, ost, opat = scene_system(bls, name, ncams, npoints)
    o = run_both(bls, st, ost, p.pattern, opat, p.E, p.C, p.R, p.b_r, p.b_e, p.scaling_r, p.scaling_e, p.lam, False, torch.float32,
                 kernel=kernel)
    assert o["ok"] and o["ook"]
    assert relerr(o["S"], o["oS"]) < 1e-4
    assert relerr(o["g"], o["og"]) < 1e-6   # z and the gradient are FP64 from FP32 data
    assert relerr(o["x_e"], o["ox_e"]) < 1e-6


@pytest.mark.parametrize("unit", [1, 3, 16, 64, 4096])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_stage_unit_sizes(bls, unit, dtype):
    """The column-owned schedule rebuilt with other unit sizes (one pair per unit up to whole blocks per unit) gives
    the same reduction, conditioning scales included."""
    p, st, ost, opat = scene_system(bls, "pcg_10000x1M", 150, 6000)
    rng = np.random.default_rng(11)
    s_r = np.ldexp(1.0, rng.integers(-4, 5, st.nr))
    s_e = np.ldexp(1.0, rng.integers(-4, 5, st.ne))
    o = run_both(bls, st, ost, p.pattern, opat, p.E, p.C, p.R, p.b_r, p.b_e, p.scaling_r, p.scaling_e, p.lam, False, dtype,
                 s_r=s_r, s_e=s_e, kernel="stage", stage_unit=unit)
    assert o["ok"] and o["ook"]
    tol = 1e-12 if dtype == torch.float64 else 1e-4
    assert relerr(o["S"], o["oS"]) < tol
    assert relerr(o["g"], o["og"]) < (1e-12 if dtype == torch.float64 else 1e-6)


def test_stage_unit_rejected(bls):
    p, st, ost, opat = scene_system(bls, "sparse_1000x200k", 40, 1500)
    ws = bls.SchurReductionWorkspace(st, p.pattern, None)
    with pytest.raises(bls.ArgumentError):
        ws.set_stage_unit(0)
    dp, dst, _, _ = scene_system(bls, "dense_50x2000", 20, 400, dense=True)
    wd = bls.SchurReductionWorkspace(dst, None, None)
    with pytest.raises(Exception, match="column-owned schedule"):
        wd.set_stage_unit(8)


@pytest.mark.parametrize("kernel", ["stage", "pairs", "points", "lanes"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("dense", [False, True])
def test_scene_conditioned_scales(bls, kernel, dtype, dense):
    """The 6/3 fast path with power-of-two conditioning scales (src/conditioning.jl:99-150) applied at read."""
    p, st, ost, opat = scene_system(bls, "sparse_1000x200k", 40, 1500, dense)
    rng = np.random.default_rng(5)
    s_r = np.ldexp(1.0, rng.integers(-4, 5, st.nr))
    s_e = np.ldexp(1.0, rng.integers(-4, 5, st.ne))
    o = run_both(bls, st, ost, p.pattern, opat, p.E, p.C, p.R, p.b_r, p.b_e, p.scaling_r, p.scaling_e, p.lam, dense, dtype,
                 s_r=s_r, s_e=s_e, kernel=kernel)
    assert o["ok"] and o["ook"]
    tol = 1e-12 if dtype == torch.float64 else 1e-4
    assert relerr(o["S"], o["oS"]) < tol
    assert relerr(o["g"], o["og"]) < (1e-12 if dtype == torch.float64 else 1e-6)


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_host_buffers_match_oracle(bls, dtype, pinned):
    """reset + reduce from host buffers, copies overlapped stage by stage, against the FP64 oracle; a singular point
    block leaves the host outputs untouched and is reported 1-based."""
    p, st, ost, opat = scene_system(bls, "sparse_1000x200k", 120, 8000, False)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    E32, C32, R32 = p.E.astype(npdt), p.C.astype(npdt), p.R.astype(npdt)

    def host(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.pin_memory() if pinned else t

    ws = bls.SchurReductionWorkspace(st, p.pattern)
    S = host(np.full(p.pattern.nnz, 7.0, npdt))
    g = host(np.full(st.nr, 7.0))
    args = [host(R32), host(p.scaling_r), p.lam, host(p.b_r), host(p.b_e), host(p.scaling_e), st, host(E32), host(C32), ws]
    assert bls.reset_reduce_schur_sparse_host(S, g, *args)
    work = orc.Work(ost, 1)
    oS, og = np.zeros(opat.nnz), np.zeros(st.nr)
    orc.reset_schur_sparse(ost, opat, oS, R32.astype(np.float64), p.scaling_r, p.lam)
    ook, _ = orc.reduce_schur_sparse(ost, opat, work, oS, og, p.b_r, p.b_e, p.scaling_e, p.lam, E32.astype(np.float64), C32.astype(np.float64))
    assert ook
    tol = 1e-12 if dtype == torch.float64 else 1e-4
    assert relerr(S.double().numpy(), oS) < tol
    assert relerr(g.numpy(), og) < (1e-12 if dtype == torch.float64 else 1e-6)
    # the same call again reproduces the result (device inputs are overwritten only after the previous call's work)
    S2, g2 = host(np.zeros(p.pattern.nnz, npdt)), host(np.zeros(st.nr))
    assert bls.reset_reduce_schur_sparse_host(S2, g2, *args)
    assert relerr(S2.double().numpy(), S.double().numpy()) < (1e-14 if dtype == torch.float64 else 1e-6)
    # point 4000 singular (its E block and damping zeroed): outputs untouched
    E_bad, sc_bad = E32.copy(), p.scaling_e.copy()
    E_bad[9 * 3999:9 * 4000] = 0.0
    sc_bad[3 * 3999:3 * 4000] = 0.0
    S3, g3 = host(np.full(p.pattern.nnz, 7.0, npdt)), host(np.full(st.nr, 7.0))
    bad = [host(R32), host(p.scaling_r), p.lam, host(p.b_r), host(p.b_e), host(sc_bad), st, host(E_bad), host(C32), ws]
    assert not bls.reset_reduce_schur_sparse_host(S3, g3, *bad)
    assert ws.failed_block == 4000
    assert (S3.numpy() == 7.0).all() and (g3.numpy() == 7.0).all()


def test_scatter_copy_matches_map(bls):
    p, st, ost, opat = scene_system(bls, "sparse_1000x200k", 60, 2000)
    colptr, rowval, smap = bls.sparse_with_map(st, p.pattern, True)
    dest = torch.empty(len(smap), dtype=torch.float64, device=DEV)
    bls.scatter_copy(dest, cu(p.R), cu(smap))
    assert np.array_equal(dest.cpu().numpy(), p.R[smap])


def test_repeated_reductions_are_stable(bls):
    """Re-running reset + reduce on the same plan gives the same S (to atomic-order rounding) every time."""
    p, st, ost, opat = scene_system(bls, "sparse_1000x200k", 120, 8000)
    ws = bls.SchurReductionWorkspace(st, p.pattern)
    outs = []
    for _ in range(3):
        S = torch.zeros(p.pattern.nnz, dtype=torch.float64, device=DEV)
        g = torch.zeros(st.nr, dtype=torch.float64, device=DEV)
        bls.reset_schur_sparse(S, cu(p.R), None, None, cu(p.scaling_r), p.lam, ws)
        assert bls.reduce_schur_sparse(S, g, cu(p.b_r), cu(p.b_e), cu(p.scaling_e), p.lam, st, cu(p.E), cu(p.C), None, None, None, None, ws)
        outs.append(S.cpu().numpy())
    for o in outs[1:]:
        assert relerr(o, outs[0]) < 1e-14


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("dense", [False, True])
def test_hessian_bilinear_and_diagonal(bls, dtype, dense):
    """dot(x, H, y) and diag(H) of the Hessian (R on the pattern or dense, E, C) against the dense H the oracle builds
    from the same stored values (FP64 sums: 1e-12 relative)."""
    p, st, ost, opat = scene_system(bls, "sparse_1000x200k", 60, 2500, dense)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    E, Cd, R = p.E.astype(npdt), p.C.astype(npdt), p.R.astype(npdt)
    ws = bls.SchurReductionWorkspace(st, p.pattern)
    if dense:
        R0 = cu(R)
        oR = R.astype(np.float64)
    else:
        R0 = torch.zeros(p.pattern.nnz, dtype=dtype, device=DEV)
        bls.reset_schur_sparse(R0, cu(R), None, None, cu(p.scaling_r), 0.0, ws)   # R on the pattern
        oR = np.zeros(opat.nnz)
        orc.reset_schur_sparse(ost, opat, oR, R.astype(np.float64), p.scaling_r, 0.0)
    H = orc.hessian_dense(ost, oR, E.astype(np.float64), Cd.astype(np.float64), None if dense else opat)
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal(H.shape[0]), rng.standard_normal(H.shape[0])
    v = ws.hessian_bilinear(R0, cu(E), cu(Cd), cu(x), cu(y), dense=dense)
    assert abs(v - x @ H @ y) <= 1e-12 * (np.abs(x) @ np.abs(H) @ np.abs(y))
    d = ws.hessian_diagonal(R0, cu(E), dense=dense)
    assert relerr(d.cpu().numpy(), np.diag(H)) <= 1e-15


@pytest.mark.parametrize("dense", [False, True])
def test_mixed_dims_mixed_form_and_failure(bls, dense):
    """Point blocks of 1 to 12 variables (mixed_dims_problem) in the mixed form against the FP64 oracle on the same
    FP32 values, and a singular 5 x 5 block reported as the lowest failing one."""
    H, b, st, ost, rr, sc = fixture_system(bls, MIXED_DIMS)
    pat = None if dense else bls.build_schur_pattern(st, rr)
    opat = None if dense else orc.Pattern(ost, rr)
    E, Cd, R = split_hessian(H, st, pat)
    nr = st.nr
    o = run_both(bls, st, ost, pat, opat, E, Cd, R, b[:nr], b[nr:], sc[:nr], sc[nr:], 0.5, dense, torch.float32)
    assert o["ok"] and o["ook"]
    assert relerr(o["S"], o["oS"]) < 1e-4 and relerr(o["g"], o["og"]) < 1e-6
    # eliminated block 7 (5 variables, 0-based 6): E and its damping zeroed
    e = 6
    eo, de, so = int(st.eoffsets[e]), int(st.e_dims[e]), int(st.boffsets_e[e])
    E2, sc2 = E.copy(), sc.copy()
    E2[eo:eo + de * de] = 0.0
    sc2[nr + so:nr + so + de] = 0.0
    o = run_both(bls, st, ost, pat, opat, E2, Cd, R, b[:nr], b[nr:], sc2[:nr], sc2[nr:], 0.5, dense, torch.float64)
    assert not o["ok"] and not o["ook"]
    assert o["fb"] == e + 1 == o["ofb"]


EDGE = {
    # a camera no point observes: its S column is its reset diagonal block, its gradient b_r
    "unobserved_camera": dict(r_dims=[6, 6, 6], e_dims=[3, 3, 3, 3], couplings=[[0, 1], [0], [1], [0, 1]]),
    # points observed by a single camera: diagonal pairs only
    "single_observations": dict(r_dims=[6, 6], e_dims=[3, 3, 3, 3, 3], couplings=[[0], [1], [0], [1], [0]]),
    # a lone point on every camera at once
    "one_point": dict(r_dims=[6, 6, 6, 6], e_dims=[3], couplings=[[0, 1, 2, 3]]),
}


@pytest.mark.parametrize("name", list(EDGE))
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "mixed"])
@pytest.mark.parametrize("dense", [False, True])
def test_edge_structures(bls, name, dtype, dense):
    """Ragged and degenerate structures on the 6/3 fast path against the oracle."""
    H, b, st, ost, rr, sc = fixture_system(bls, EDGE[name])
    pat = None if dense else bls.build_schur_pattern(st, rr)
    opat = None if dense else orc.Pattern(ost, rr)
    E, Cd, R = split_hessian(H, st, pat)
    nr = st.nr
    o = run_both(bls, st, ost, pat, opat, E, Cd, R, b[:nr], b[nr:], sc[:nr], sc[nr:], 0.5, dense, dtype)
    assert o["ok"] and o["ook"]
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    assert relerr(o["S"], o["oS"]) < tol and relerr(o["g"], o["og"]) < 1e-12


def test_plan_needs_an_eliminated_block(bls):
    """A structure without eliminated blocks has nothing to reduce: the device plan rejects it (ArgumentError) instead
    of returning the reset system as the reference's loop over no blocks does."""
    st = bls.SchurStructure.positional([6, 6], [], [])
    pat = bls.build_schur_pattern(st, [])
    with pytest.raises(bls.ArgumentError, match="at least one retained and one eliminated block"):
        bls.SchurReductionWorkspace(st, pat)
