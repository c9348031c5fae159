"""The product's native QR layout (SchurJacobianStructure) against the oracle: bit-exact integers.

Covers the description constructor (src/schur_description.jl:137-189: tables of eliminated blocks, free groups numbered
by first appearance, row placement) and the positional one (src/schur_jacobian.jl:59-160) on the reference's QR test
structures (test/fixtures/QRFixtures.jl:55-80), the doctest and known answers (src/schur_description.jl:129-134,
test/qr_reduction.jl:176-178), random descriptions with free rows, and the seeded QR workload scaled down.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from qr_fixtures import QR_FIXTURES

KA = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())

QR_FIELDS = ("table_nrows", "table_ncols", "table_top", "table_offsets", "raw_offsets", "residual_offsets", "reduced_offsets",
             "table_ptr", "entry_retained", "entry_col", "entry_table", "retained_ptr", "retained_entry", "doffsets", "e_rows",
             "free_rows", "col_chunks")
ROW_FIELDS = ("row_table", "row_first", "row_nrows", "row_ptr", "row_blocks")


def _same_qr(j, o, rows=False):
    assert j.ntables == o.ntables
    for f in QR_FIELDS:
        np.testing.assert_array_equal(getattr(j, f), getattr(o, f), err_msg=f)
    assert j.raw_length == o.raw_length and j.residual_length == o.residual_length
    if rows:
        for f in ROW_FIELDS:
            np.testing.assert_array_equal(getattr(j, f), o.field(f), err_msg=f)
    for f in ("r_dims", "e_dims", "eliminated_ptr", "entry_retained", "order", "boffsets_r", "boffsets_e"):
        np.testing.assert_array_equal(getattr(j.schur, f), getattr(o.st, f), err_msg="schur." + f)


def test_doctest_jacobian_structure(bls):
    c = KA["doctest_jacobian_structure"]
    j = bls.SchurJacobianStructure(c["blocksizes"], c["rowblocks"], c["rowblocksizes"], eliminated=c["eliminated"])
    assert list(j.blockorder()) == c["blockorder"] and j.nretained() == c["nretained"] and j.nblocks() == c["nblocks"]
    o = orc.QRStructure.from_description(c["blocksizes"], c["rowblocks"], c["rowblocksizes"], c["eliminated"])
    _same_qr(j, o, rows=True)


def test_free_group_known_answer(bls):
    c = KA["qr_free_group"]
    j = bls.SchurJacobianStructure(c["blocksizes"], c["rowblocks"], c["rowblocksizes"], eliminated=c["eliminated"])
    assert j.ntables == c["ntables"] and list(j.free_rows) == c["free_rows"]
    _same_qr(j, orc.QRStructure.from_description(c["blocksizes"], c["rowblocks"], c["rowblocksizes"], c["eliminated"]), rows=True)


def test_qr_bytes_known_answer(bls):
    c = KA["qr_bytes"]
    st = bls.SchurStructure.positional([6] * c["nret"], [3] * c["nelim"], [list(range(c["nret"]))] * c["nelim"])
    j = bls.SchurJacobianStructure.positional(st, [c["rows"]] * c["nelim"])
    assert 2 * 8 * (j.raw_length + j.residual_length) == c["expected_bytes"]


@pytest.mark.parametrize("name", list(QR_FIXTURES))
@pytest.mark.parametrize("nchunks", [1, 3])
def test_positional_fixtures(bls, name, nchunks):
    fx = QR_FIXTURES[name](np.random.default_rng(1))
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"], nchunks=nchunks)
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"], nchunks=nchunks)
    j = bls.SchurJacobianStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()), nchunks=nchunks)
    o = orc.QRStructure.positional(ost, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()), nchunks=nchunks)
    _same_qr(j, o)
    if name == "free groups":
        assert bls.free_block_pairs(j) == [(0, 1), (1, 3), (1, 4), (3, 4)]


def _random_qr_description(rng, n_ret, n_el):
    n = n_ret + n_el
    perm = rng.permutation(n)
    bs = np.empty(n, np.int64)
    el = np.zeros(n, bool)
    bs[perm[:n_ret]] = rng.choice([6, 3, 9], n_ret)
    bs[perm[n_ret:]] = rng.choice([3, 2, 1, 4], n_el)
    el[perm[n_ret:]] = True
    rbs, sizes = [], []
    for e in range(n_el):
        for _ in range(rng.integers(1, 4)):
            k = rng.integers(0, min(3, n_ret) + 1)
            rbs.append([int(perm[n_ret + e])] + [int(perm[c]) for c in rng.choice(n_ret, k, replace=False)])
            sizes.append(int(rng.integers(1, 4)))
    for _ in range(rng.integers(0, 2 * n_ret)):   # free rows, some groups repeated
        k = rng.integers(1, min(3, n_ret) + 1)
        rbs.append([int(perm[c]) for c in rng.choice(n_ret, k, replace=False)])
        sizes.append(int(rng.integers(1, 3)))
    order = rng.permutation(len(rbs))
    return bs, el, [rbs[i] for i in order], [sizes[i] for i in order]


@pytest.mark.parametrize("seed", range(6))
def test_random_descriptions(bls, seed):
    rng = np.random.default_rng(500 + seed)
    bs, el, rbs, sizes = _random_qr_description(rng, int(rng.integers(1, 8)), int(rng.integers(1, 30)))
    for nchunks in (1, 4):
        j = bls.SchurJacobianStructure(bs, rbs, sizes, eliminated=el, nchunks=nchunks)
        o = orc.QRStructure.from_description(bs, rbs, sizes, el, nchunks=nchunks)
        _same_qr(j, o, rows=True)


def test_scene_layout(bls):
    spec = bls.scenes.scaled_down(bls.scenes.workload("qr_500x100k"), ncams=40, npoints=800)
    p = bls.scenes.jacobian_problem(spec)
    sc = bls.scenes.Scene(spec)
    bs, el, ptr, idx = sc.description()
    o = orc.QRStructure.from_description(bs, (ptr, idx), np.full(len(ptr) - 1, 2), el)
    _same_qr(p.structure, o, rows=True)
    # every observation's two rows landed in its point's table: the data rows of each table are filled
    j = p.structure
    for t in range(0, j.schur.neblocks, 97):
        M, C = int(j.table_nrows[t]), int(j.table_ncols[t]) - 1
        T = p.Rw[j.raw_offsets[t]:j.raw_offsets[t + 1]].reshape(C, M).T
        me = M - int(j.table_top[t])
        assert np.all(T[:me, C - 3:] != 0) and np.all(T[me:] == 0)


def test_rejected(bls):
    # every row block needs at least one row; an eliminated block needs rows (src/schur_description.jl:38-64)
    with pytest.raises(bls.ArgumentError, match="Row block 2 has 0 rows"):
        bls.SchurJacobianStructure([6, 3], [[0, 1], [0]], [2, 0], eliminated=[False, True])
    with pytest.raises(bls.ArgumentError, match="Eliminated column block 3 is in no row block"):
        bls.SchurJacobianStructure([6, 3, 3], [[0, 1]], [2], eliminated=[False, True, True])
    with pytest.raises(bls.DimensionMismatch):
        bls.SchurJacobianStructure([6, 3], [[0, 1]], [2, 2], eliminated=[False, True])
    st = bls.SchurStructure.positional([6, 6], [3], [[0, 1]])
    with pytest.raises(bls.ArgumentError):
        bls.SchurJacobianStructure.positional(st, [0])
    with pytest.raises(bls.ArgumentError):
        bls.SchurJacobianStructure.positional(st, [2], [3], [[0, 0]])
    with pytest.raises(bls.DimensionMismatch):
        bls.SchurJacobianStructure.positional(st, [2, 2])


def _reduced_pattern_checks(bls, j, o):
    colptr, rowval = bls.build_reduced_jacobian_pattern(j)
    ocp, orv = orc.reduced_jacobian_pattern(o)
    np.testing.assert_array_equal(colptr, ocp)
    np.testing.assert_array_equal(rowval, orv)
    # nnz(J~) = sum over entries of d_r of its retained block times the reduced rows of its table (test/schur_qr.jl:243-245)
    nnz = sum(int(j.schur.r_dims[j.entry_retained[u]]) * int(j.table_nrows[j.entry_table[u]] - j.table_top[j.entry_table[u]])
              for u in range(len(j.entry_retained)))
    assert len(rowval) == nnz == colptr[-1]
    assert colptr.shape == (j.schur.nr + 1,) and np.all(np.diff(colptr) >= 0)
    assert np.all((rowval >= 0) & (rowval < bls.reduced_nrows(j)))


@pytest.mark.parametrize("name", list(QR_FIXTURES))
def test_reduced_jacobian_pattern_fixtures(bls, name):
    """build_reduced_jacobian_pattern (src/qr_reduced.jl:284-310): the native host pattern equals the oracle's."""
    fx = QR_FIXTURES[name](np.random.default_rng(3))
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    j = bls.SchurJacobianStructure.positional(st, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    o = orc.QRStructure.positional(ost, fx["e_rows"], fx.get("free_rows", ()), fx.get("free_retained", ()))
    _reduced_pattern_checks(bls, j, o)


def test_reduced_jacobian_pattern_scene(bls):
    spec = bls.scenes.scaled_down(bls.scenes.workload("qr_500x100k"), ncams=40, npoints=800)
    p = bls.scenes.jacobian_problem(spec)
    sc = bls.scenes.Scene(spec)
    bs, el, ptr, idx = sc.description()
    o = orc.QRStructure.from_description(bs, (ptr, idx), np.full(len(ptr) - 1, 2), el)
    _reduced_pattern_checks(bls, p.structure, o)
