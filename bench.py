"""Benchmark: observations/s through the Schur reduction of the pcg_10000x1M scene (10,000 cameras, 1,000,000 points,
~7.7M observations), then block-Jacobi PCG on the reduced system to 1e-8, on N GPUs as N independent replicas (the
reduction has no cross-GPU exchange).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one reset_schur_sparse + reduce_schur_sparse of the whole scene. `value` is the mixed form (FP32 storage
and accumulation, FP64 point-block inverse, z and gradient) with inputs resident in device memory, L2 flushed
between steps; `fp64` reports the plain FP64 form the same way. `e2e` runs the same step through the public API from
pinned host buffers: one reset_reduce_schur_sparse_host call per step, which copies the inputs in stage by stage while
the earlier stages are reduced and copies S and g_S out. The roofline is the phase-2 kernel's: the algorithmic bytes
of the reduction (per point 84 + 76 k bytes in the mixed form, plus one read and one write of S), over its
event-timed duration, against the measured HBM copy bandwidth. `pcg` adds seconds to ||g - S x|| <= 1e-8 ||g||
(FP64 residual) on the mixed S, and the refined solve against the FP64 reduced operator to 1e-10. The CPU-baseline
leg runs the oracle's FP64 reduction of the same scene and reports the device results' distance from it (`parity`).

--impl reference times the reference algorithm (the oracle: a C++ restatement of BlockLinearSystems.jl's
reset_schur_sparse! + reduce_schur_sparse!, threaded over its chunks as the reference threads over Polyester chunks)
on every host core, in FP64: the reference's Float32 path rejects this scene's point blocks as singular. Its inputs
are generated by a separate, untimed child process and read back from .npy files, so the timed process loads no
library of this repository.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path
from types import SimpleNamespace

import numpy as np

ROOT = Path(__file__).resolve().parent
METRIC = "observations/s through Schur reduction, mixed vs FP64 plain; PCG s to 1e-8"


def load_package():
    import importlib.util
    name = "blsgpu"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "blocklinearsystems.jl_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def algorithmic_bytes(p, dtype_bytes: int) -> float:
    """Bytes the reduction must move: per point 9 E + 18k C entries in the storage type, b_e and scaling_e (FP64), a
    4-byte camera index per observation; plus S read and written once."""
    st = p.structure
    per_point = dtype_bytes * (9 * st.neblocks + 18 * p.nobs) + 8 * (3 + 3) * st.neblocks + 4 * p.nobs
    return float(per_point + 2 * dtype_bytes * p.pattern.nnz)


def algorithmic_flops(p) -> float:
    """F(k) = 58 + 270 k + 108 k (k - 1) per point (FMA = 2)."""
    st = p.structure
    k = np.diff(st.eliminated_ptr).astype(np.float64)
    return float((58 + 270 * k + 108 * k * (k - 1)).sum())


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest of every rank's x (a job's time is its slowest replica's); x itself on one rank."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_spec(spec, rank: int, world: int):
    """Each replica's own scene: the same distribution, the seed moved by 100 per rank (one rank keeps it)."""
    if world == 1:
        return spec
    from dataclasses import replace
    return replace(spec, seed=spec.seed + 100 * rank)


L2_NOTE = "flushed between timed steps (256 MB write)"
SCHUR_STEP = "reset_schur_sparse + reduce_schur_sparse"
QR_STEP = "reduce_qr + reduced_normal_sparse"


def hessian_config(workload: str, world: int, cameras: int, points: int, observations: int, nnz_S: int) -> dict:
    """The `config` both arms print for a Hessian workload (the reference arm reads the numbers from its fixture)."""
    return {"workload": workload, "cameras": int(cameras), "points": int(points), "observations": int(observations),
            "nnz_S": int(nnz_S), "parallelism": f"replicas x{world}", "l2": L2_NOTE, "step": SCHUR_STEP}


def qr_config(workload: str, world: int, cameras: int, points: int, observations: int, table_entries: int, nnz_S: int) -> dict:
    return {"workload": workload, "cameras": int(cameras), "points": int(points), "observations": int(observations),
            "table_entries": int(table_entries), "nnz_S": int(nnz_S), "parallelism": f"replicas x{world}", "l2": L2_NOTE,
            "step": QR_STEP}


def dense_config(workload: str, world: int, cameras: int, points: int, n: int) -> dict:
    return {"workload": workload, "cameras": int(cameras), "points": int(points), "n": int(n),
            "step": "bls_dense_cholesky + bls_dense_cholesky_solve", "l2": "S (288 MB) larger than L2",
            "parallelism": f"replicas x{world}"}


def batch_config(workload: str, world: int, problems: int, cameras: int, points: int, observations: int, nnz_S: int) -> dict:
    return {"workload": workload, "problems": int(problems), "cameras": int(cameras), "points": int(points),
            "observations": int(observations), "nnz_S": int(nnz_S), "parallelism": f"replicas x{world}", "l2": L2_NOTE,
            "step": "one CUDA graph replay: reset_schur_sparse + reduce_schur_sparse of all problems (disjoint-union plan)"}


def measured_traffic(workload: str, kernel: str) -> float | None:
    """DRAM read + write bytes per launch of `kernel` on `workload`, from one ncu capture summarised under profiles/
    (traffic_<workload>.json, keyed by kernel name); None when no capture of that kernel on that workload exists."""
    f = ROOT / "profiles" / f"traffic_{workload}.json"
    if not f.exists():
        return None
    rec = json.loads(f.read_text()).get(kernel)
    return None if rec is None else rec.get("dram_bytes_per_launch")


def schur_parity(S_orc: np.ndarray, g_orc: np.ndarray, results: dict) -> dict:
    """Distance of the device results from the oracle's FP64 reduction of the same scene: ||S - S_oracle|| /
    ||S_oracle|| and the same for g_S, per form, against the tolerances the tests use (1e-12 FP64, 1e-4 mixed)."""
    out = {"reference": "oracle FP64 reset_schur_sparse + reduce_schur_sparse of the same inputs (the CPU-baseline run)"}
    ok = True
    ns, ng = float(np.linalg.norm(S_orc)), float(np.linalg.norm(g_orc))
    for name, (S, g, tol) in results.items():
        es = float(np.linalg.norm(S.astype(np.float64) - S_orc)) / ns
        eg = float(np.linalg.norm(g - g_orc)) / ng
        out[name] = {"S_rel": es, "g_rel": eg, "tol": tol}
        ok = ok and es <= tol and eg <= tol
    out["ok"] = ok
    return out


def run_ours(args, rank: int, world: int) -> dict | None:
    import torch
    bls = load_package()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    spec = bls.scenes.workload(args.workload)
    spec = replica_spec(spec, rank, world)   # each replica its own scene of the same distribution
    p = bls.scenes.hessian_problem(spec)
    st, pat = p.structure, p.pattern
    ws = bls.SchurReductionWorkspace(st, pat, device=dev.index)
    if args.schedule:
        ws.set_kernel(args.schedule)
    if args.stage_unit:
        ws.set_stage_unit(args.stage_unit)
    flush = torch.empty(256 * 2**20 // 4, dtype=torch.float32, device=dev)   # larger than the 126 MB L2

    def device_inputs(dt):
        f = lambda a, t=dt: torch.from_numpy(a).to(device=dev, dtype=t)
        return dict(E=f(p.E), C=f(p.C), R=f(p.R), b_r=f(p.b_r, torch.float64), b_e=f(p.b_e, torch.float64),
                    sr=f(p.scaling_r, torch.float64), se=f(p.scaling_e, torch.float64),
                    S=torch.zeros(pat.nnz, dtype=dt, device=dev), g=torch.zeros(st.nr, dtype=torch.float64, device=dev))

    def step(d):
        bls.reset_schur_sparse(d["S"], d["R"], None, None, d["sr"], p.lam, ws)
        bls.reduce_schur_sparse(d["S"], d["g"], d["b_r"], d["b_e"], d["se"], p.lam, st, d["E"], d["C"], None, None, None, None, ws,
                                sync=False)

    def timed(d, steps, warmup, instrument=False):
        for _ in range(warmup):
            step(d)
        assert ws.query_status(), f"reduction failed at block {ws.failed_block}"
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ws.instrument(instrument)
        ws.counters()
        total = 0.0
        evs = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            step(d)
            b.record()
            evs.append((a, b))
        torch.cuda.synchronize()
        total = sum(a.elapsed_time(b) for a, b in evs)
        cnt = ws.counters()
        ws.instrument(False)
        ok = ws.query_status()
        assert ok, f"reduction failed at block {ws.failed_block}"
        total = max_over_ranks(total, world, dev)
        return total, cnt

    d32 = device_inputs(torch.float32)
    with ClockSampler(dev.index) as clk:
        ms32, cnt32 = timed(d32, args.steps, args.warmup, instrument=True)
    _LAST.update(problem=p, d32=d32, ws=ws, step=step)
    S32h, g32h = d32["S"].cpu().numpy(), d32["g"].cpu().numpy()   # the last timed step's results (parity below)
    d64 = device_inputs(torch.float64)
    ms64, cnt64 = timed(d64, args.steps, args.warmup, instrument=True)
    S64h, g64h = d64["S"].cpu().numpy(), d64["g"].cpu().numpy()
    del d64

    # end to end through the public API from pinned host buffers (mixed form)
    host = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in
            dict(E=p.E.astype(np.float32), C=p.C.astype(np.float32), R=p.R.astype(np.float32), b_r=p.b_r, b_e=p.b_e,
                 sr=p.scaling_r, se=p.scaling_e).items()}
    S_host = torch.empty(pat.nnz, dtype=torch.float32).pin_memory()
    g_host = torch.empty(st.nr, dtype=torch.float64).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    d2h = S_host.numel() * 4 + g_host.numel() * 8

    def e2e_step():
        # one public call on host buffers: the library overlaps the stage-by-stage copies with the reduction and
        # copies S and g_S back (synchronous; asserts the verdict)
        assert bls.reset_reduce_schur_sparse_host(S_host, g_host, host["R"], host["sr"], p.lam, host["b_r"], host["b_e"], host["se"],
                                                  st, host["E"], host["C"], ws)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        e2e_step()
    b.record()
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b)
    e2e_ms = max_over_ranks(e2e_ms, world, dev)
    assert ws.query_status()

    if rank != 0:
        return None
    nobs = p.nobs
    value = world * nobs * args.steps / (ms32 / 1e3)
    v64 = world * nobs * args.steps / (ms64 / 1e3)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    pair_ms = cnt32["pair_kernel_ms"] / max(cnt32["pair_kernel_launches"], 1)
    bytes32 = algorithmic_bytes(p, 4)
    achieved = bytes32 / (pair_ms / 1e3) / 1e9
    kernel = ws.phase2_kernel_name(torch.float32)
    out = {
        "metric": METRIC, "value": value, "unit": "obs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 storage/accumulation + f64 point inverse, z, gradient", "data": "synthetic (seeded scene generator)",
        "config": hessian_config(args.workload, world, st.nrblocks, st.neblocks, nobs, pat.nnz),
        "fp64": {"value": v64, "unit": "obs/s", "ms_per_step": ms64 / args.steps,
                 "phase2_kernel_ms": cnt64["pair_kernel_ms"] / max(cnt64["pair_kernel_launches"], 1),
                 "phase2_kernel": ws.phase2_kernel_name(torch.float64)},
        "mixed_over_fp64": value / v64,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": measured_traffic(args.workload, kernel), "kernel": kernel, "kernel_ms": pair_ms,
                     "stage_unit": args.stage_unit or "20 (FP32) / 16 (FP64)",
                     "algorithmic_bytes": bytes32, "peak_source": "measured" if peaks else "fallback",
                     "flops": algorithmic_flops(p), "achieved_tflops": algorithmic_flops(p) / (pair_ms / 1e3) / 1e12},
        "e2e": {"value": world * nobs * args.steps / (e2e_ms / 1e3), "unit": "obs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": cnt32["launches"],
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        view = hessian_view(bls, spec, p)
        base, S_orc, g_orc = cpu_baseline(view, seconds=args.cpu_seconds)
        _LAST.update(view=view, oracle_S=S_orc, oracle_g=g_orc)
        out["cpu_baseline"] = base
        out["parity"] = schur_parity(S_orc, g_orc, {"fp64": (S64h, g64h, 1e-12), "mixed": (S32h, g32h, 1e-4)})
    return out


def qr_algorithmic_bytes(jst, dtype_bytes: int) -> float:
    """Bytes reduce_qr must move: every raw table read and its factored copy written in the storage type, every residual
    row read and written in FP64, scaling_e read (FP64)."""
    cells = float(np.sum(jst.table_nrows * (jst.table_ncols - 1)))
    rows = float(np.sum(jst.table_nrows))
    return 2 * dtype_bytes * cells + 2 * 8 * rows + 8 * jst.schur.ne


def run_ours_qr(args, rank: int, world: int) -> dict | None:
    """The QR workload: a step is reduce_qr of every table plus reduced_normal_sparse (J~'J~ and J~'r~ on the pattern)."""
    import torch
    bls = load_package()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    spec = bls.scenes.workload(args.workload)
    spec = replica_spec(spec, rank, world)
    p = bls.scenes.jacobian_problem(spec)
    jst = p.structure
    pat = bls.build_schur_pattern(jst.schur, bls.free_block_pairs(jst))
    flush = torch.empty(256 * 2**20 // 4, dtype=torch.float32, device=dev)
    sc_e = torch.from_numpy(p.scaling_e).to(dev)

    def setup(dt):
        ws = bls.QRReductionWorkspace(jst, pat, dt, device=dev.index)
        J = bls.SchurBlockJacobian(jst, dt, device=dev.index, data=torch.from_numpy(p.Rw).to(device=dev, dtype=dt),
                                   r=torch.from_numpy(p.Rr).to(dev))
        S = torch.zeros(pat.nnz, dtype=dt, device=dev)
        g = torch.zeros(jst.schur.nr, dtype=torch.float64, device=dev)
        return ws, J, S, g

    def timed(ws, J, S, g):
        for _ in range(args.warmup):
            bls.reduce_qr(ws, J, sc_e, p.lam, sync=False)
            bls.reduced_normal_sparse(S, g, ws, pat)
        assert ws.query_status(), f"reduce_qr failed at block {ws.failed_block}"
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ws.launches()
        evs = []
        for _ in range(args.steps):
            flush.zero_()
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record()
            bls.reduce_qr(ws, J, sc_e, p.lam, sync=False)
            b.record()
            bls.reduced_normal_sparse(S, g, ws, pat)
            c.record()
            evs.append((a, b, c))
        torch.cuda.synchronize()
        launches = ws.launches()
        assert ws.query_status()
        total = sum(a.elapsed_time(c) for a, b, c in evs)
        qr_ms = sum(a.elapsed_time(b) for a, b, c in evs) / args.steps
        total = max_over_ranks(total, world, dev)
        return total, qr_ms, launches

    ws32, J32, S32, g32 = setup(torch.float32)
    with ClockSampler(dev.index) as clk:
        ms32, qr32, launches = timed(ws32, J32, S32, g32)
    ws64, J64, S64, g64 = setup(torch.float64)
    ms64, qr64, _ = timed(ws64, J64, S64, g64)
    del ws64, J64, S64, g64

    # end to end from pinned host buffers: raw tables (FP32) and residual in, J~'J~ and J~'r~ out
    hRw = torch.from_numpy(p.Rw.astype(np.float32)).pin_memory()
    hRr = torch.from_numpy(p.Rr).pin_memory()
    hS = torch.empty(pat.nnz, dtype=torch.float32).pin_memory()
    hg = torch.empty(jst.schur.nr, dtype=torch.float64).pin_memory()

    def e2e_step():
        J32.data.copy_(hRw, non_blocking=True)
        J32.r.copy_(hRr, non_blocking=True)
        bls.reduce_qr(ws32, J32, sc_e, p.lam, sync=False)
        bls.reduced_normal_sparse(S32, g32, ws32, pat)
        hS.copy_(S32, non_blocking=True)
        hg.copy_(g32, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        e2e_step()
    b.record()
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b)
    assert ws32.query_status()

    # the Hessian route from the same Jacobian: assemble H = J'J, b = J'r on the device (FP32 tables, FP64 sums), then
    # the mixed Schur reduction of it (R reset from the pattern through the identity map); the assembly alone and the
    # whole route, per step
    sws = bls.SchurReductionWorkspace(jst.schur, pat, r_to_s_map=np.arange(pat.nnz), device=dev.index)
    Sh = torch.zeros(pat.nnz, dtype=torch.float32, device=dev)
    gh = torch.zeros(jst.schur.nr, dtype=torch.float64, device=dev)
    zr = torch.zeros(jst.schur.nr, dtype=torch.float64, device=dev)
    nr = jst.schur.nr

    def hess_step(mid=None):
        E, Cd, R, bb = bls.assemble_hessian(J32, ws32)
        if mid is not None:
            mid.record()
        bls.reset_schur_sparse(Sh, R, None, None, zr, p.lam, sws)
        bls.reduce_schur_sparse(Sh, gh, bb[:nr], bb[nr:], sc_e, p.lam, jst.schur, E, Cd, None, None, None, None, sws, sync=False)

    for _ in range(args.warmup):
        hess_step()
    assert sws.query_status()
    asm_ms, route_ms = [], []
    for _ in range(args.steps):
        flush.zero_()
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record()
        hess_step(b)
        c.record()
        torch.cuda.synchronize()
        asm_ms.append(a.elapsed_time(b))
        route_ms.append(a.elapsed_time(c))
    assert sws.query_status()
    asm = statistics.median(asm_ms)
    # the matrix-free LSMR solve of the reduced problem (block-Jacobi preconditioned; the reference's Krylov extension)
    # on the mixed tables: at the reference's tolerances for Float32 storage, and at 1e-10; wall time of the
    # synchronous call, median of three
    assert bls.reduce_qr(ws32, J32, sc_e, p.lam)
    xr = torch.zeros(nr, dtype=torch.float64, device=dev)
    lsmr = {}
    for name, kw in (("tol_sqrt_eps_f32", {}), ("tol_1e-10", dict(atol=1e-10, btol=1e-10, conlim=1e14))):
        res = bls.lsmr_reduced(xr, ws32, p.lam, **kw)
        walls = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = bls.lsmr_reduced(xr, ws32, p.lam, **kw)
            walls.append((time.perf_counter() - t0) * 1e3)
        ms = statistics.median(walls)
        lsmr[name] = {"ms": ms, "iterations": res.iterations, "istop": res.istop, "solved": res.solved,
                      "ms_per_iteration": ms / max(res.iterations, 1)}
    # the bound of an iteration: J~ read twice (J~ t and J~' u; the retained columns of every table's reduced rows)
    n_red = (np.asarray(jst.table_nrows) - np.asarray(jst.table_top)).astype(np.int64)
    ent_tab = np.repeat(np.arange(jst.ntables), np.diff(np.asarray(jst.table_ptr)))
    jt_bytes = int(np.sum(n_red[ent_tab] * np.asarray(jst.schur.r_dims)[np.asarray(jst.entry_retained)])) * 4
    a_, b_ = lsmr["tol_sqrt_eps_f32"], lsmr["tol_1e-10"]
    if b_["iterations"] > a_["iterations"]:
        per_it = (b_["ms"] - a_["ms"]) / (b_["iterations"] - a_["iterations"])
        lsmr["per_iteration"] = {"ms": per_it, "jt_bytes_f32": jt_bytes, "achieved_gbs": 2 * jt_bytes / (per_it / 1e3) / 1e9,
                                 "note": "wall ms per extra iteration (two host read-backs included) over two passes of J~"}
    st_ = jst.schur
    asm_bytes = int(jst.raw_length * 4 + jst.residual_length * 8 + (st_.E_length + st_.C_length + pat.nnz) * 4 + (st_.nr + st_.ne) * 8)
    if rank != 0:
        return None
    nobs = p.nobs
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    b32 = qr_algorithmic_bytes(jst, 4)
    achieved = b32 / (qr32 / 1e3) / 1e9
    prof = ROOT / "profiles" / "qr_tables_qr_500x100k.json"
    traffic = json.loads(prof.read_text()).get("dram_bytes_per_launch_f32") if prof.exists() else None
    out = {
        "metric": METRIC, "value": world * nobs * args.steps / (ms32 / 1e3), "unit": "obs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 tables + f64 norms, reflector arithmetic, residual", "data": "synthetic (seeded scene generator)",
        "config": {"workload": args.workload, "cameras": jst.schur.nrblocks, "points": jst.schur.neblocks, "observations": nobs,
                   "table_entries": int(np.sum(jst.table_nrows * (jst.table_ncols - 1))), "nnz_S": pat.nnz,
                   "parallelism": f"replicas x{world}", "l2": "flushed between timed steps (256 MB write)",
                   "step": "reduce_qr + reduced_normal_sparse"},
        "fp64": {"value": world * nobs * args.steps / (ms64 / 1e3), "unit": "obs/s", "ms_per_step": ms64 / args.steps, "reduce_qr_ms": qr64},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                     "kernel": "reduce_qr (k_qr_tables<float>)", "kernel_ms": qr32, "algorithmic_bytes": b32,
                     "peak_source": "measured" if peaks else "fallback"},
        "e2e": {"value": world * nobs * args.steps / (e2e_ms / 1e3), "unit": "obs/s",
                "h2d_bytes_per_step": hRw.numel() * 4 + hRr.numel() * 8, "d2h_bytes_per_step": hS.numel() * 4 + hg.numel() * 8},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "hessian_route": {"assemble_ms": asm, "assemble_gbs": asm_bytes / (asm / 1e3) / 1e9, "assemble_frac": asm_bytes / (asm / 1e3) / 1e9 / hbm,
                          "assemble_bytes": asm_bytes, "ms_per_step": statistics.median(route_ms),
                          "obs_per_s": nobs / (statistics.median(route_ms) / 1e3),
                          "step": "assemble_hessian (J'J, J'r from the f32 tables) + mixed reset_schur_sparse + reduce_schur_sparse"},
        "lsmr": dict(lsmr, step="lsmr_reduced on the mixed factored tables, lambda of the workload, s_r = 1"),
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_qr(jacobian_view(bls, spec, p), seconds=args.cpu_seconds)
    return out


def cpu_baseline_qr(v, seconds: float = 10.0, steps: int | None = None, warmup: int = 1) -> dict:
    """The reference algorithm (oracle) on every host core, FP64: reduce_qr threaded over its chunks, then
    reduced_normal_sparse threaded over retained block columns, as the reference threads them."""
    orc = oracle_module()
    cores = os.cpu_count() or 1
    o = orc.QRStructure.from_description(v.bs, (v.ptr, v.idx), np.full(len(v.ptr) - 1, 2), v.el, nchunks=cores)
    opat = orc.Pattern(o.st)
    F, Fr = np.zeros(o.raw_length), np.zeros(o.residual_length)
    S, g = np.zeros(opat.nnz), np.zeros(o.st.nr)

    def one():
        ok, _ = orc.reduce_qr(o, F, Fr, v.Rw, v.Rr, v.scaling_e, v.lam, nthreads=cores)
        assert ok
        orc.reduced_normal_sparse(o, opat, S, g, F, Fr)

    for _ in range(warmup):
        one()
    n, t0 = 0, time.perf_counter()
    while (steps is None and (time.perf_counter() - t0 < seconds or n < 3)) or (steps is not None and n < steps):
        one()
        n += 1
    dt = time.perf_counter() - t0
    return {"value": v.nobs * n / dt, "unit": "obs/s", "cores": cores, "kind": "port",
            "sample": f"{n} x full reduce_qr + reduced_normal_sparse of {int(v.el.sum())} points / {v.nobs} observations, FP64, "
                      f"{cores} OpenMP threads ({dt:.1f} s)"}


def run_ours_pcg(args, rank: int, world: int) -> dict | None:
    """The PCG workload: the mixed reduction of the scene (timed as the Schur workload is), then PCG on the mixed S to
    ||g - S x|| <= 1e-8 ||g|| (FP64 residual), block-Jacobi preconditioned; seconds per solve on the device."""
    import torch
    out = run_ours(args, rank, world)
    bls = load_package()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    p = _LAST["problem"]
    st, pat, d32 = p.structure, p.pattern, _LAST["d32"]
    pws = bls.PCGWorkspace(st, pat, device=dev.index)
    S, g = d32["S"], d32["g"]
    x = torch.zeros(st.nr, dtype=torch.float64, device=dev)
    times, iters, rels = [], [], []
    for k in range(args.warmup + args.steps):
        x.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record()
        _, res = pws.solve(S, g, x, tol=1e-8)
        b.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        assert res.converged, res
        if k >= args.warmup:
            times.append((a.elapsed_time(b) / 1e3, wall))
            iters.append(res.iterations)
            rels.append(res.rel_residual)
    pws.launches()
    if rank != 0:
        return None
    dev_s = statistics.median(t[0] for t in times)
    out["pcg"] = {"seconds_to_1e-8": dev_s, "wall_seconds": statistics.median(t[1] for t in times), "iterations": iters[-1],
                  "rel_residual": rels[-1], "preconditioner": "block-Jacobi (6x6)", "S_storage": "f32 (mixed reduction output)",
                  "residual": "explicit FP64 g - S x"}
    # the learned block preconditioner (trained by blocklinearsystems.jl_b200/train_gnn.py on the 1k-5k-camera scenes of
    # this workload's family) against block-Jacobi on this scene: iterations and device seconds to 1e-8, the learned side
    # including its BF16 inference of the blocks
    pfile = ROOT / "blocklinearsystems.jl_b200" / "gnn_pcg_params.npy"
    if pfile.exists():
        net = bls.gnn.LearnedPreconditioner(pws)
        assert net.prepare(S)
        params = torch.from_numpy(np.load(pfile)).to(dev)
        for _ in range(args.warmup):
            bls.gnn.pcg_comparison(net, S, g, params)
        cmp_ = bls.gnn.pcg_comparison(net, S, g, params)
        if rank == 0:
            out["pcg"]["learned"] = dict(cmp_, target="learned time <= 0.6 x block-Jacobi",
                                         params=f"{pfile.name}, trained by train_gnn.py (summary in {pfile.with_suffix('.json').name})")
        del net
    # the same solve refined against the FP64 reduced operator (R + lambda D - C' E^-1 C applied from the stored blocks
    # and the reduction's FP64 E^-1) to 1e-10: PCG corrections on the FP32 S, outer residual in FP64
    ws = _LAST["ws"]
    _LAST["step"](d32)
    assert ws.query_status()
    S0 = torch.zeros_like(S)
    bls.reset_schur_sparse(S0, d32["R"], None, None, d32["sr"], 0.0, ws)
    rtimes = []
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        _, rres = pws.solve_refined(S, S0, d32["sr"], p.lam, d32["C"], g, ws, x, tol=1e-10, inner_tol=1e-6)
        b.record()
        torch.cuda.synchronize()
        assert rres.converged, rres
        if k >= args.warmup:
            rtimes.append(a.elapsed_time(b) / 1e3)
    out["pcg"]["refined"] = {"seconds_to_1e-10": statistics.median(rtimes), "corrections": rres.corrections,
                             "iterations": rres.iterations, "rel_residual": rres.rel_residual,
                             "residual": "FP64 g - A x, A = R + lambda D - C' E^-1 C from the stored blocks",
                             "inner": "PCG on the f32 S to 1e-6 per correction"}
    if not args.no_cpu_baseline:
        out["pcg"]["cpu_baseline"] = cpu_baseline_pcg(_LAST["view"], _LAST["oracle_S"], _LAST["oracle_g"])
    return out


def dense_launches(n: int) -> tuple[int, int]:
    """Kernels one dense factorisation and one solve launch for an n x n system (64-column panels; a panel with at most
    32 tiles below it is one launch, otherwise its diagonal tile and its rows are two)."""
    panels = (n + 63) // 64
    panel_kernels = 0
    for k in range(panels):
        nb = min(64, n - 64 * k)
        below = (n - 64 * k - nb + 63) // 64
        panel_kernels += 1 if below <= 32 else 2
    factor = 1 + panel_kernels + (panels - 1) + max(panels - 2, 0)   # load, panels, next-panel updates, the rest
    solve = 2 * panels   # a forward step per tile, the last tile and a backward step per other tile
    return factor, solve


def run_ours_dense(args, rank: int, world: int) -> dict | None:
    """The dense reduced solve: reduce_schur_dense! of the scene into a dense FP64 S (6 variables per camera), then a
    step is the device Cholesky of S plus one solve x = S^-1 g (the reference's cholesky(Symmetric(S)) \\ g); S, 288 MB
    for 1,000 cameras, is larger than L2. The roofline is FP64 over the whole factorisation against cuBLAS DGEMM measured
    in the same run (no FP64 peak is measured for the pool)."""
    import torch
    bls = load_package()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    spec = replica_spec(bls.scenes.workload(args.workload), rank, world)
    p = bls.scenes.hessian_problem(spec, dense=True)
    st = p.structure
    n = st.nr
    f = lambda a, t=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=t)
    ws = bls.SchurReductionWorkspace(st, None, device=dev.index)
    S = torch.zeros(n * n, dtype=torch.float64, device=dev)
    g = torch.zeros(n, dtype=torch.float64, device=dev)
    bls.reset_schur_dense(S, f(p.R), f(p.scaling_r), p.lam, ws)
    assert bls.reduce_schur_dense(S, g, f(p.b_r), f(p.b_e), f(p.scaling_e), p.lam, st, f(p.E), f(p.C), ws)
    del ws
    D = bls.DenseCholesky(n, device=dev.index)
    x = torch.empty_like(g)

    def step():
        assert D.factor(S), f"S is not positive definite (column {D.failed_column})"
        D.solve(g, x)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    evs = []
    with ClockSampler(dev.index) as clk:
        for _ in range(args.steps):
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record()
            assert D.factor(S)
            b.record()
            D.solve(g, x)
            c.record()
            evs.append((a, b, c))
        torch.cuda.synchronize()
    total = max_over_ranks(sum(a.elapsed_time(c) for a, _, c in evs), world, dev)
    factor_ms = statistics.median(a.elapsed_time(b) for a, b, _ in evs)
    solve_ms = statistics.median(b.elapsed_time(c) for _, b, c in evs)
    A = S.view(n, n).t()   # S is column-major: A[i, j] = S[i + n j]; its upper triangle is the reduced system
    Afull = torch.triu(A) + torch.triu(A, 1).t()
    rel = float((Afull @ x - g).norm() / g.norm())
    del Afull, A

    # end to end through the public API: S and g from pinned host memory, x back to the host
    S_host = S.cpu().pin_memory()
    g_host = g.cpu().pin_memory()
    x_host = torch.empty(n, dtype=torch.float64).pin_memory()
    S_dev = torch.empty_like(S)
    g_dev = torch.empty_like(g)

    def e2e_step():
        S_dev.copy_(S_host, non_blocking=True)
        g_dev.copy_(g_host, non_blocking=True)
        assert D.factor(S_dev)
        D.solve(g_dev, x)
        x_host.copy_(x, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        e2e_step()
    b.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(a.elapsed_time(b), world, dev)
    assert torch.equal(x_host, x.cpu())

    # the FP64 denominator: cuBLAS DGEMM (torch.matmul, float64, 8192^3), best of 3
    M = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    M @ M
    best = float("inf")
    for _ in range(3):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        M @ M
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    dgemm_tflops = 2 * 8192**3 / (best / 1e3) / 1e12
    del M
    if rank != 0:
        return None
    fl, sl = dense_launches(n)
    flops = n**3 / 3.0
    achieved = flops / (factor_ms / 1e3) / 1e12
    out = {
        "metric": "dense reduced solves/s (Cholesky of the dense S + one solve)", "value": world * args.steps / (total / 1e3),
        "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene generator)",
        "config": {"workload": args.workload, "cameras": st.nrblocks, "points": st.neblocks, "n": n,
                   "step": "bls_dense_cholesky + bls_dense_cholesky_solve", "l2": "S (288 MB) larger than L2",
                   "parallelism": f"replicas x{world}"},
        "factor_ms": factor_ms, "solve_ms": solve_ms, "rel_residual": rel,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": dgemm_tflops, "unit": "TFLOP/s", "frac": achieved / dgemm_tflops,
                     "traffic": None, "scope": "whole factorisation (n^3 / 3 multiply-adds as flops over its event time)",
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (torch.matmul, float64)"},
        "e2e": {"value": world * args.steps / (e2e_ms / 1e3), "unit": "solves/s", "h2d_bytes_per_step": n * n * 8 + n * 8,
                "d2h_bytes_per_step": n * 8},
        "gpu_launches": args.steps * (fl + sl),
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_dense(S_host.numpy(), g_host.numpy(), n, seconds=args.cpu_seconds)
    return out


def dense_reduced_host(v):
    """The dense S and g of the scene from the oracle's reset_schur_dense + reduce_schur_dense (FP64, every host core)."""
    cores = os.cpu_count() or 1
    orc, ost, _ = oracle_structure(v, cores)
    n = ost.nr
    S, g = np.zeros(n * n), np.zeros(n)
    orc.reset_schur_dense(ost, S, v.R, v.scaling_r, v.lam)
    ok, _ = orc.reduce_schur_dense(ost, orc.Work(ost, cores, False), S, g, v.b_r, v.b_e, v.scaling_e, v.lam, v.E, v.C, nthreads=cores)
    assert ok
    return S, g


def cpu_baseline_dense(S: np.ndarray, g: np.ndarray, n: int, seconds: float = 10.0, steps: int | None = None) -> dict:
    """LAPACK dpotrf + dpotrs (scipy, every host core) on the same S: the routine the reference's
    cholesky(Symmetric(S)) \\ g reaches."""
    import scipy.linalg as sl
    A = np.asarray(S, np.float64).reshape(n, n, order="F")
    cores = os.cpu_count() or 1

    def one():
        c = sl.cho_factor(A, lower=False, overwrite_a=False, check_finite=False)
        return sl.cho_solve(c, g, check_finite=False)

    one()
    k, t0 = 0, time.perf_counter()
    while (steps is None and (time.perf_counter() - t0 < seconds or k < 3)) or (steps is not None and k < steps):
        one()
        k += 1
    dt = time.perf_counter() - t0
    return {"value": k / dt, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"{k} x LAPACK dpotrf + dpotrs of the {n} x {n} S through scipy on {cores} host threads ({dt:.1f} s)"}


_LAST: dict = {}


def run_ours_batch(args, rank: int, world: int) -> dict | None:
    """The batched workload: 256 independent problems of uneven sizes, each with its own lambda, reduced as one plan
    over the disjoint union of their layouts; a step is one replay of the CUDA graph holding reset + reduce of the whole
    batch (mixed form), with the phase-2 schedule picked by the autotuner."""
    import torch
    bls = load_package()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    nprob = 256
    problems = []
    for i in range(nprob):
        spec = bls.scenes.workload(args.workload, i + (1000 * rank if world > 1 else 0))
        problems.append(bls.scenes.hessian_problem(spec))
    flush = torch.empty(256 * 2**20 // 4, dtype=torch.float32, device=dev)

    def timed(B):
        for _ in range(args.warmup):
            B.step()
        assert B.ok()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        B.ws.counters()
        evs = []
        for _ in range(args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            B.step()
            b.record()
            evs.append((a, b))
        torch.cuda.synchronize()
        assert B.ok()
        total = sum(a.elapsed_time(b) for a, b in evs)
        total = max_over_ranks(total, world, dev)
        return total

    B64 = bls.batch.BatchedReduction(problems, torch.float64, device=dev.index)
    tunes64 = B64.autotune()
    B64.capture()
    ms64 = timed(B64)
    S64 = B64.S.cpu().numpy()
    del B64
    B = bls.batch.BatchedReduction(problems, torch.float32, device=dev.index)
    tunes = B.autotune()
    B.ws.counters()
    B.run(sync=False)
    per_step = B.ws.counters()["launches"]   # the kernels one step launches (the graph holds the same kernels)
    B.capture()
    with ClockSampler(dev.index) as clk:
        ms32 = timed(B)
    # per-problem error of the mixed result against the FP64 reduction of the same problem (FP64 inputs)
    S32 = B.S.double().cpu().numpy()
    errs = []
    for i in range(nprob):
        a, b = int(B.off["nnz"][i]), int(B.off["nnz"][i + 1])
        errs.append(float(np.linalg.norm(S32[a:b] - S64[a:b]) / np.linalg.norm(S64[a:b])))
    # end to end: every input from pinned host memory, S and g back
    host = {k: getattr(B, k).cpu().pin_memory() for k in ("E", "C", "R", "b_r", "b_e", "sc_r", "sc_e")}
    hS = torch.empty_like(B.S, device="cpu").pin_memory()
    hg = torch.empty_like(B.g, device="cpu").pin_memory()

    def e2e_step():
        # one public call on host buffers over the batch's union plan (copies overlapped with the reduction)
        assert B.run_host(hS, hg, host)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        e2e_step()
    b.record()
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b)
    assert B.ok()
    if rank != 0:
        return None
    nobs = B.nobs
    out = {
        "metric": METRIC, "value": world * nobs * args.steps / (ms32 / 1e3), "unit": "obs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 storage/accumulation + f64 point inverse, z, gradient", "data": "synthetic (seeded scene generator)",
        "config": {"workload": args.workload, "problems": nprob, "cameras": int(B.U.nrblocks), "points": int(B.U.neblocks),
                   "observations": nobs, "nnz_S": int(B.U.nnz), "parallelism": f"replicas x{world}",
                   "l2": "flushed between timed steps (256 MB write)",
                   "step": "one CUDA graph replay: reset_schur_sparse + reduce_schur_sparse of all problems (disjoint-union plan)"},
        "schedule": {"chosen": B.schedule + (f"/{B.stage_unit}" if B.schedule == "stage" else ""), "autotune_ms": tunes, "fp64_chosen": min(tunes64, key=tunes64.get), "fp64_autotune_ms": tunes64},
        "fp64": {"value": world * nobs * args.steps / (ms64 / 1e3), "unit": "obs/s", "ms_per_step": ms64 / args.steps},
        "per_problem_error_vs_fp64": {"max": max(errs), "median": float(np.median(errs)), "norm": "||S_mixed - S_fp64|| / ||S_fp64|| per problem"},
        "e2e": {"value": world * nobs * args.steps / (e2e_ms / 1e3), "unit": "obs/s",
                "h2d_bytes_per_step": int(sum(v.numel() * v.element_size() for v in host.values())),
                "d2h_bytes_per_step": int(hS.numel() * 4 + hg.numel() * 8)},
        "gpu_launches": per_step * args.steps,
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_batch([hessian_view(bls, p.spec, p) for p in problems], seconds=args.cpu_seconds)
    return out


def cpu_baseline_batch(views, seconds: float = 10.0) -> dict:
    """The reference algorithm (oracle) on every host core, FP64: each problem reset + reduced in turn."""
    orc = oracle_module()
    cores = os.cpu_count() or 1
    prepared = []
    for v in views:
        _, ost, opat = oracle_structure(v, cores)
        prepared.append((v, ost, opat, orc.Work(ost, cores, False), np.zeros(opat.nnz), np.zeros(ost.nr)))
    n, nobs, t0 = 0, 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds or n < 1:
        for v, ost, opat, w, S, g in prepared:
            orc.reset_schur_sparse(ost, opat, S, v.R, v.scaling_r, v.lam)
            ok, _ = orc.reduce_schur_sparse(ost, opat, w, S, g, v.b_r, v.b_e, v.scaling_e, v.lam, v.E, v.C, nthreads=cores)
            assert ok
            nobs += v.nobs
        n += 1
    dt = time.perf_counter() - t0
    return {"value": nobs / dt, "unit": "obs/s", "cores": cores, "kind": "port",
            "sample": f"{n} x all {len(views)} problems reset + reduced in turn, FP64, {cores} OpenMP threads ({dt:.1f} s)"}


def cpu_baseline_pcg(v, S: np.ndarray, g: np.ndarray) -> dict:
    """The oracle's PCG (the same algorithm on every host core) on the oracle's FP64 reduced system of the same scene."""
    orc = oracle_module()
    _, ost, opat = oracle_structure(v, os.cpu_count() or 1)
    cores = os.cpu_count() or 1
    x = np.zeros(ost.nr)
    t0 = time.perf_counter()
    rc, it, rel = orc.pcg_solve(ost, opat, S, g, x, 1e-8, nthreads=cores)
    dt = time.perf_counter() - t0
    return {"seconds_to_1e-8": dt, "iterations": it, "rel_residual": rel, "cores": cores, "kind": "port",
            "sample": f"one block-Jacobi PCG solve to 1e-8, FP64, {cores} OpenMP threads"}


# --- the inputs of a workload as plain numpy arrays ------------------------------------------------------------------
# Both arms hand the oracle a "view": the scene's description (blocksizes, eliminated flags, row-block pointers and
# indices) and its assembled arrays. The repository arm builds it from its own problem; the reference arm reads it from
# .npy files that a separate, untimed child process wrote, so that the timed reference process maps no library of
# this repository (only numpy and the oracle).
HESSIAN_ARRAYS = ("bs", "el", "ptr", "idx", "E", "C", "R", "b_r", "b_e", "scaling_r", "scaling_e")
JACOBIAN_ARRAYS = ("bs", "el", "ptr", "idx", "Rw", "Rr", "scaling_e")


def hessian_view(bls, spec, p) -> SimpleNamespace:
    bs, el, ptr, idx = bls.scenes.Scene(spec).description()
    return SimpleNamespace(bs=bs, el=el, ptr=ptr, idx=idx, E=p.E, C=p.C, R=p.R, b_r=p.b_r, b_e=p.b_e, scaling_r=p.scaling_r,
                           scaling_e=p.scaling_e, lam=float(p.lam), nobs=int(p.nobs))


def jacobian_view(bls, spec, p) -> SimpleNamespace:
    bs, el, ptr, idx = bls.scenes.Scene(spec).description()
    return SimpleNamespace(bs=bs, el=el, ptr=ptr, idx=idx, Rw=p.Rw, Rr=p.Rr, scaling_e=p.scaling_e, lam=float(p.lam),
                           nobs=int(p.nobs))


def _save_view(d: Path, v: SimpleNamespace, names) -> None:
    d.mkdir(parents=True, exist_ok=True)
    for k in names:
        a = getattr(v, k)
        np.save(d / f"{k}.npy", np.ascontiguousarray(a.astype(np.uint8) if k == "el" else a))
    (d / "scalars.json").write_text(json.dumps({"lam": v.lam, "nobs": v.nobs}))


def _load_view(d: Path, names) -> SimpleNamespace:
    v = SimpleNamespace(**{k: np.load(d / f"{k}.npy") for k in names})
    v.el = v.el.astype(bool)
    sc = json.loads((d / "scalars.json").read_text())
    v.lam, v.nobs = float(sc["lam"]), int(sc["nobs"])
    return v


def write_fixture(workload: str, out: Path) -> None:
    """Generate the workload with this repository's scene generator and write the reference arm's inputs and the
    numbers of its `config` (run in a child process by --impl reference)."""
    bls = load_package()
    out.mkdir(parents=True, exist_ok=True)
    if workload.startswith("batched_"):
        nprob, sums = 256, dict(cameras=0, points=0, observations=0, nnz_S=0)
        for i in range(nprob):
            spec = bls.scenes.workload(workload, i)
            p = bls.scenes.hessian_problem(spec)
            _save_view(out / f"p{i:03d}", hessian_view(bls, spec, p), HESSIAN_ARRAYS)
            sums["cameras"] += p.structure.nrblocks
            sums["points"] += p.structure.neblocks
            sums["observations"] += p.nobs
            sums["nnz_S"] += p.pattern.nnz
        meta = dict(kind="batch", problems=nprob, **sums)
    elif workload.startswith("qr_"):
        spec = bls.scenes.workload(workload)
        p = bls.scenes.jacobian_problem(spec)
        jst = p.structure
        pat = bls.build_schur_pattern(jst.schur, bls.free_block_pairs(jst))
        _save_view(out, jacobian_view(bls, spec, p), JACOBIAN_ARRAYS)
        meta = dict(kind="qr", cameras=jst.schur.nrblocks, points=jst.schur.neblocks, observations=p.nobs,
                    table_entries=int(np.sum(jst.table_nrows * (jst.table_ncols - 1))), nnz_S=pat.nnz)
    else:
        spec = bls.scenes.workload(workload)
        dense = workload.startswith("dense_")
        p = bls.scenes.hessian_problem(spec, dense=dense)
        _save_view(out, hessian_view(bls, spec, p), HESSIAN_ARRAYS)
        st = p.structure
        meta = dict(kind="dense" if dense else "hessian", cameras=st.nrblocks, points=st.neblocks, observations=p.nobs,
                    n=st.nr, nnz_S=0 if dense else p.pattern.nnz)
    (out / "meta.json").write_text(json.dumps(meta))


def oracle_module():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    return orc


def oracle_structure(v, cores: int):
    orc = oracle_module()
    ost = orc.Structure.from_description(v.bs, (v.ptr, v.idx), v.el, nchunks=cores, min_work=4096)
    return orc, ost, orc.Pattern(ost)


def cpu_baseline(v, seconds: float = 10.0, steps: int | None = None, warmup: int = 1):
    """The reference algorithm (oracle) on every host core, FP64, reset + reduce of the scene in `v`; returns the
    baseline record and the oracle's S and g_S of its last run."""
    cores = os.cpu_count() or 1
    orc, ost, opat = oracle_structure(v, cores)
    w = orc.Work(ost, cores, False)
    S = np.zeros(opat.nnz)
    g = np.zeros(ost.nr)

    def one():
        orc.reset_schur_sparse(ost, opat, S, v.R, v.scaling_r, v.lam)
        ok, _ = orc.reduce_schur_sparse(ost, opat, w, S, g, v.b_r, v.b_e, v.scaling_e, v.lam, v.E, v.C, nthreads=cores)
        assert ok

    for _ in range(warmup):
        one()
    n, t0 = 0, time.perf_counter()
    while (steps is None and (time.perf_counter() - t0 < seconds or n < 3)) or (steps is not None and n < steps):
        one()
        n += 1
    dt = time.perf_counter() - t0
    base = {"value": v.nobs * n / dt, "unit": "obs/s", "cores": cores, "kind": "port",
            "sample": f"{n} x full reset_schur_sparse + reduce_schur_sparse of {int(v.el.sum())} points / {v.nobs} "
                      f"observations, FP64, {cores} OpenMP threads over the reference's chunks ({dt:.1f} s)"}
    return base, S, g


def reference_line(args, world: int, base: dict, config: dict, metric: str = METRIC, unit: str = "obs/s",
                   dtype: str = "f64") -> dict:
    # the time of one step of the workload at the measured rate (observations per step, or one solve)
    per_step = config.get("observations", 1) if unit == "obs/s" else 1
    ms = 1e3 * per_step / base["value"] if base["value"] else None
    return {"impl": "reference", "metric": metric, "value": base["value"], "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded scene generator)", "config": config,
            "note": "reference algorithm restated in C++ (the oracle; Julia is unavailable); inputs read from .npy files "
                    "written by an untimed child process",
            "cpu_baseline": base, "e2e": {"value": base["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference(args, rank: int, world: int) -> dict | None:
    if rank != 0:
        return None
    import shutil
    import tempfile
    tmp = Path(tempfile.mkdtemp(prefix="bls_ref_"))
    try:
        subprocess.run([sys.executable, str(Path(__file__).resolve()), "--write-fixture", str(tmp), "--workload", args.workload],
                       check=True)
        meta = json.loads((tmp / "meta.json").read_text())
        if meta["kind"] == "batch":
            views = [_load_view(tmp / f"p{i:03d}", HESSIAN_ARRAYS) for i in range(meta["problems"])]
            shutil.rmtree(tmp, ignore_errors=True)
            base = cpu_baseline_batch(views, seconds=args.cpu_seconds)
            cfg = batch_config(args.workload, world, meta["problems"], meta["cameras"], meta["points"], meta["observations"],
                               meta["nnz_S"])
            return reference_line(args, world, base, cfg)
        if meta["kind"] == "qr":
            v = _load_view(tmp, JACOBIAN_ARRAYS)
            shutil.rmtree(tmp, ignore_errors=True)
            base = cpu_baseline_qr(v, steps=args.steps, warmup=args.warmup)
            cfg = qr_config(args.workload, world, meta["cameras"], meta["points"], meta["observations"], meta["table_entries"],
                            meta["nnz_S"])
            return reference_line(args, world, base, cfg)
        v = _load_view(tmp, HESSIAN_ARRAYS)
        shutil.rmtree(tmp, ignore_errors=True)
        if meta["kind"] == "dense":
            S, g = dense_reduced_host(v)
            base = cpu_baseline_dense(S, g, meta["n"], steps=args.steps)
            cfg = dense_config(args.workload, world, meta["cameras"], meta["points"], meta["n"])
            return reference_line(args, world, base, cfg, metric="dense reduced solves/s (Cholesky of the dense S + one solve)",
                                  unit="solves/s")
        base, S, g = cpu_baseline(v, steps=args.steps, warmup=args.warmup)
        cfg = hessian_config(args.workload, world, meta["cameras"], meta["points"], meta["observations"], meta["nnz_S"])
        out = reference_line(args, world, base, cfg)
        if args.workload.startswith("pcg_"):
            out["pcg"] = cpu_baseline_pcg(v, S, g)
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pcg_10000x1M")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stage-unit", type=int, default=None, help="pairs per unit of the column-owned schedule (default 16)")
    ap.add_argument("--schedule", default=None, help="phase-2 schedule of the Schur workloads (default: the plan's, stage)")
    ap.add_argument("--write-fixture", default=None, help=argparse.SUPPRESS)   # the reference arm's untimed child
    args = ap.parse_args()
    if args.write_fixture:
        write_fixture(args.workload, Path(args.write_fixture))
        return
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world)
        elif args.workload.startswith("qr_"):
            out = run_ours_qr(args, rank, world)
        elif args.workload.startswith("pcg_"):
            out = run_ours_pcg(args, rank, world)
        elif args.workload.startswith("batched_"):
            out = run_ours_batch(args, rank, world)
        elif args.workload.startswith("dense_"):
            out = run_ours_dense(args, rank, world)
        else:
            out = run_ours(args, rank, world)
    finally:
        if world > 1 and args.impl == "ours":
            import torch
            torch.distributed.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
