"""Seeded synthetic bundle-adjustment workloads (no public dataset is named for this path).

Each workload has the stated shape and distributions; the generator (csrc/scene.cpp) uses splitmix64-seeded
xoshiro256** streams, one per point, with seed = 1000 * workload number + problem index.

  dense_50x2000       50 cameras, 2,000 points, k ~ U{2..8} from all cameras, lambda 1e-3, dense retained part
  sparse_1000x200k    1,000 cameras, 200,000 points, window +-30, k = 2 + Geom(0.2) capped at 40, point singular
                      values log-uniform in [1e-4, 1], lambda 1e-4
  qr_500x100k         500 cameras, 100,000 points, window +-20, k = 2 + Geom(0.2) capped at 16, point singular values
                      log-uniform in [1e-7, 1], lambda 1e-6 (damping rows sqrt(lambda) I)
  batched_256         256 problems, cameras U{10..400}, points U{1,000..50,000}, window +-15, k = 2 + Geom(0.3)
                      capped at 20, lambda log-uniform in [1e-6, 1e-2] per problem
  pcg_10000x1M        10,000 cameras, 1,000,000 points, window +-60, k = 2 + Geom(0.15) capped at 60, camera column
                      scales log-uniform in [1e-2, 1e2], lambda 1e-5
  dense_1000x200k     sparse_1000x200k's distributions with its own seed, reduced into a dense S (6,000 x 6,000)
Damping is Marquardt's, lambda * diag(H), for every Hessian workload.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, replace

import numpy as np

from . import _lib
from ._lib import ptr64
from .layout import SchurPattern, SchurStructure, build_schur_pattern


@dataclass(frozen=True)
class SceneSpec:
    ncams: int
    npoints: int
    covis: str = "window"          # "uniform" or "window"
    kmin: int = 2
    kmax: int = 8
    geom_p: float = 0.2
    kcap: int = 40
    window: int = 30
    sv: tuple | None = None        # point-Jacobian singular values, log-uniform (lo, hi)
    cs: tuple | None = None        # camera column scales, log-uniform (lo, hi)
    lam: float = 1e-4
    seed: int = 0


def workload(name: str, problem: int = 0) -> SceneSpec:
    """The named workload's spec (problem indexes the batched workload's problems)."""
    if name == "dense_50x2000":
        return SceneSpec(50, 2000, "uniform", 2, 8, lam=1e-3, seed=1000 * 1 + problem)
    if name == "sparse_1000x200k":
        return SceneSpec(1000, 200_000, "window", geom_p=0.2, kcap=40, window=30, sv=(1e-4, 1.0), lam=1e-4, seed=1000 * 2 + problem)
    if name == "qr_500x100k":
        return SceneSpec(500, 100_000, "window", geom_p=0.2, kcap=16, window=20, sv=(1e-7, 1.0), lam=1e-6, seed=1000 * 3 + problem)
    if name == "batched_256":
        rng = np.random.Generator(np.random.PCG64(4000 + problem))
        nc = int(rng.integers(10, 401))
        npnt = int(rng.integers(1000, 50_001))
        lam = float(math.exp(rng.uniform(math.log(1e-6), math.log(1e-2))))
        return SceneSpec(nc, npnt, "window", geom_p=0.3, kcap=20, window=15, lam=lam, seed=1000 * 4 + problem)
    if name == "dense_1000x200k":
        return SceneSpec(1000, 200_000, "window", geom_p=0.2, kcap=40, window=30, sv=(1e-4, 1.0), lam=1e-4, seed=1000 * 6 + problem)
    if name == "pcg_10000x1M":
        return SceneSpec(10_000, 1_000_000, "window", geom_p=0.15, kcap=60, window=60, cs=(1e-2, 1e2), lam=1e-5, seed=1000 * 5 + problem)
    raise KeyError(name)


def scaled_down(spec: SceneSpec, ncams: int, npoints: int, seed: int | None = None) -> SceneSpec:
    """The same distributions on fewer cameras and points (for tests the oracle finishes in seconds)."""
    return replace(spec, ncams=ncams, npoints=npoints, window=min(spec.window, max(1, ncams // 2)),
                   seed=spec.seed if seed is None else seed)


class Scene:
    """A generated scene: per observation a camera, a 2x6 camera Jacobian, a 2x3 point Jacobian and a residual."""

    def __init__(self, spec: SceneSpec):
        L = _lib.scene_lib()
        self.spec = spec
        h = C.c_void_p()
        covis = 0 if spec.covis == "uniform" else 1
        sv_lo, sv_hi = spec.sv if spec.sv else (0.0, 0.0)
        cs_lo, cs_hi = spec.cs if spec.cs else (0.0, 0.0)
        rc = L.bls_scene_generate(spec.ncams, spec.npoints, covis, spec.kmin, spec.kmax, spec.geom_p, spec.kcap, spec.window,
                                  sv_lo, sv_hi, cs_lo, cs_hi, spec.seed, C.byref(h))
        if rc != 0:
            raise ValueError("bad scene spec")
        self._h = h
        self.ncams = int(L.bls_scene_size(h, 0))
        self.npoints = int(L.bls_scene_size(h, 1))
        self.nobs = int(L.bls_scene_size(h, 2))

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None and _lib._scene is not None:
            _lib.scene_lib().bls_scene_destroy(self._h)
            self._h = None

    def arrays(self):
        """(obs_ptr, obs_cam, Jc[nobs,6,2]->column-major 2x6, Jp, r) as numpy arrays."""
        L = _lib.scene_lib()
        obs_ptr = np.empty(self.npoints + 1, np.int64)
        obs_cam = np.empty(self.nobs, np.int64)
        Jc = np.empty(self.nobs * 12)
        Jp = np.empty(self.nobs * 6)
        r = np.empty(self.nobs * 2)
        dp = C.POINTER(C.c_double)
        L.bls_scene_arrays(self._h, ptr64(obs_ptr), ptr64(obs_cam), Jc.ctypes.data_as(dp), Jp.ctypes.data_as(dp), r.ctypes.data_as(dp))
        return obs_ptr, obs_cam, Jc.reshape(self.nobs, 6, 2), Jp.reshape(self.nobs, 3, 2), r.reshape(self.nobs, 2)

    def description(self):
        """(blocksizes, eliminated, rowblock_ptr, rowblock_idx): cameras 0..ncams-1 then points; one row block
        [camera, point] per observation."""
        L = _lib.scene_lib()
        n = self.ncams + self.npoints
        bs = np.empty(n, np.int64)
        el = np.empty(n, np.uint8)
        ptr = np.empty(self.nobs + 1, np.int64)
        idx = np.empty(2 * self.nobs, np.int64)
        L.bls_scene_description(self._h, ptr64(bs), el.ctypes.data_as(C.POINTER(C.c_uint8)), ptr64(ptr), ptr64(idx))
        return bs, el.astype(bool), ptr, idx


@dataclass
class HessianProblem:
    """A scene assembled as H = J'J, b = J'r in the reference's SchurBlockHessian layout (float64 host arrays)."""
    spec: SceneSpec
    structure: SchurStructure
    pattern: SchurPattern | None
    dense: bool
    E: np.ndarray
    C: np.ndarray
    R: np.ndarray          # dense: column-major nr*nr; sparse: the retained storage on the pattern
    b_r: np.ndarray
    b_e: np.ndarray
    scaling_r: np.ndarray
    scaling_e: np.ndarray
    lam: float
    nobs: int
    extra: dict = field(default_factory=dict)


def hessian_problem(spec: SceneSpec, *, dense: bool = False, nchunks: int = 1, min_work: int = 4096) -> HessianProblem:
    """Generate a scene, lay it out with SchurStructure(blocksizes, rowblocks; eliminated) and assemble J'J and J'r into
    E_data, C_data, R and b (addblock!, src/schur_assembly.jl:140-246). Damping scaling: diag(H) (Marquardt)."""
    sc = Scene(spec)
    bs, el, ptr, idx = sc.description()
    st = SchurStructure(bs, (ptr, idx), eliminated=el, nchunks=nchunks, min_work=min_work)
    pat = None if dense else build_schur_pattern(st)
    nr, ne = st.nr, st.ne
    E = np.empty(st.E_length)
    Cd = np.empty(st.C_length)
    if dense:
        R = np.empty(nr * nr)
        R_diag = None
        R_dense_nr = nr
    else:
        R = np.empty(pat.R_length)
        R_diag = np.ascontiguousarray(pat.R_diag_start(st.nrblocks))
        R_dense_nr = 0
    b_r = np.empty(nr)
    b_e = np.empty(ne)
    position = np.ascontiguousarray(st.position())
    dp = C.POINTER(C.c_double)
    _lib.scene_lib().bls_scene_assemble(sc._h, ptr64(position), ptr64(st.eliminated_ptr), ptr64(st.entry_retained), ptr64(st.coffsets),
                                        ptr64(st.eoffsets), ptr64(st.boffsets_r), ptr64(st.boffsets_e), R_dense_nr,
                                        ptr64(R_diag) if R_diag is not None else None, E.ctypes.data_as(dp), len(E),
                                        Cd.ctypes.data_as(dp), len(Cd), R.ctypes.data_as(dp), len(R), b_r.ctypes.data_as(dp), nr,
                                        b_e.ctypes.data_as(dp), ne)
    # Marquardt damping scaling: the diagonal of H
    scaling_e = np.empty(ne)
    for e_dim in np.unique(st.e_dims):
        sel = np.nonzero(st.e_dims == e_dim)[0]
        for i in range(int(e_dim)):
            scaling_e[st.boffsets_e[sel] + i] = E[st.eoffsets[sel] + i * (int(e_dim) + 1)]
    if dense:
        scaling_r = R.reshape(nr, nr, order="F").diagonal().copy()
    else:
        scaling_r = np.empty(nr)
        for r in range(st.nrblocks):
            d = int(st.r_dims[r])
            for i in range(d):
                scaling_r[st.boffsets_r[r] + i] = R[R_diag[r] + i * (d + 1)]
    return HessianProblem(spec, st, pat, dense, E, Cd, R, b_r, b_e, scaling_r, scaling_e, spec.lam, sc.nobs)


@dataclass
class JacobianProblem:
    """A scene laid out as the reference's SchurBlockJacobian: one row block [camera, point] of 2 rows per observation,
    the raw tables (float64) and the residual (float64) in the structure's layout, damping sqrt(lambda * scaling_e) with
    scaling_e = 1 (the plain sqrt(lambda) I damping rows)."""
    spec: SceneSpec
    structure: "object"    # qr.SchurJacobianStructure
    Rw: np.ndarray
    Rr: np.ndarray
    scaling_e: np.ndarray
    lam: float
    nobs: int


def jacobian_problem(spec: SceneSpec, *, nchunks: int = 1, min_work: int = 4096) -> JacobianProblem:
    """Generate a scene, lay it out with SchurJacobianStructure(blocksizes, rowblocks, rowblocksizes; eliminated) and
    write each observation's camera and point Jacobians and residual into its table (src/schur_jacobian.jl:368-387)."""
    from .qr import SchurJacobianStructure
    sc = Scene(spec)
    bs, el, ptr, idx = sc.description()
    rbs = np.full(len(ptr) - 1, 2, np.int64)
    jst = SchurJacobianStructure(bs, (ptr, idx), rbs, eliminated=el, nchunks=nchunks, min_work=min_work)
    Rw = np.empty(jst.raw_length)
    Rr = np.empty(jst.residual_length)
    position = np.ascontiguousarray(jst.schur.position())
    dp = C.POINTER(C.c_double)
    rc = _lib.scene_lib().bls_scene_assemble_qr(sc._h, ptr64(position), ptr64(jst.row_table), ptr64(jst.row_first), ptr64(jst.table_ptr),
                                                ptr64(jst.entry_retained), ptr64(jst.entry_col), ptr64(jst.table_nrows),
                                                ptr64(jst.table_ncols), ptr64(jst.raw_offsets), ptr64(jst.residual_offsets),
                                                Rw.ctypes.data_as(dp), len(Rw), Rr.ctypes.data_as(dp), len(Rr))
    if rc != 0:
        raise ValueError("the scene does not match the structure")
    return JacobianProblem(spec, jst, Rw, Rr, np.ones(jst.schur.ne), spec.lam, sc.nobs)
