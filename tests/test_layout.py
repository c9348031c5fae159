"""The product's native host layout (libblsgpu) against the oracle: bit-exact integers.

Covers SchurStructure from a description and positionally, build_schur_pattern (with extra blocks), the block-level
r -> s map, the workspace index and column chunks, and makesparseindices / sparse_with_map, on the reference's test
structures, seeded scenes of every workload family, and random descriptions with several block sizes and retained pairs.
Also the rejected descriptions and their messages (test/schur_description.jl:66-90).
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from fixtures import COUPLED_GROUPS, GAUGE, SCHUR_JL, STANDARD

KA = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())

STRUCT_FIELDS = ("r_dims", "e_dims", "boffsets_r", "boffsets_e", "eoffsets", "eliminated_ptr", "entry_retained", "coffsets", "order")


def _same_structure(st, o):
    assert st.nr == o.nr and st.nrblocks == o.nrblocks and st.neblocks == o.neblocks and st.max_coupled_dim == o.max_coupled_dim
    for f in STRUCT_FIELDS:
        np.testing.assert_array_equal(getattr(st, f), getattr(o, f), err_msg=f)
    np.testing.assert_array_equal(st.retained_pairs.ravel(), o.retained_pairs, err_msg="retained_pairs")
    np.testing.assert_array_equal(st.chunks, o.chunks, err_msg="chunks")


def _same_pattern(bls, st, ost, extra=()):
    p = bls.build_schur_pattern(st, extra)
    q = orc.Pattern(ost, extra)
    for f in orc.Pattern.FIELDS:
        np.testing.assert_array_equal(getattr(p, f), getattr(q, f), err_msg=f)
    assert p.R_length == q.R_length
    np.testing.assert_array_equal(bls.build_r_to_s_map(st, p), q.r_to_s_map())
    for sym in (False, True):
        a = bls.sparse_with_map(st, p, sym)
        b = q.sparse_indices(sym)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    return p


def _same_workspace(st, ost, nchunks):
    w = orc.Work(ost, nchunks)
    for f in ("retained_ptr", "retained_entry", "entry_eliminated", "col_chunks"):
        np.testing.assert_array_equal(getattr(st, f), w.field(f), err_msg=f)


@pytest.mark.parametrize("fx", [SCHUR_JL, STANDARD, COUPLED_GROUPS, GAUGE], ids=["schur_jl", "standard", "coupled_groups", "gauge"])
@pytest.mark.parametrize("nchunks", [1, 3, 4])
def test_positional_fixtures(bls, fx, nchunks):
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"], nchunks=nchunks)
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"], nchunks=nchunks)
    _same_structure(st, ost)
    _same_workspace(st, ost, nchunks)
    _same_pattern(bls, st, ost, fx.get("rr_pairs", ()))


def test_docstring_layout(bls):
    c = KA["doctest_structure"]
    st = bls.SchurStructure(c["blocksizes"], c["rowblocks"], eliminated=c["eliminated"])
    assert list(st.blockorder()) == c["blockorder"] and st.nretained() == c["nretained"]
    assert list(st.blocksizes()) == c["layout_blocksizes"]


def _random_description(rng, n_ret, n_el, rowblocks_per_el, with_retained_rows):
    sizes_r = rng.choice([6, 3, 9], n_ret)
    sizes_e = rng.choice([3, 2, 1], n_el)
    n = n_ret + n_el
    perm = rng.permutation(n)   # caller numbering differs from the layout's
    bs = np.empty(n, np.int64)
    el = np.zeros(n, bool)
    bs[perm[:n_ret]] = sizes_r
    bs[perm[n_ret:]] = sizes_e
    el[perm[n_ret:]] = True
    rbs = []
    for e in range(n_el):
        for _ in range(rng.integers(1, rowblocks_per_el + 1)):
            k = rng.integers(1, min(4, n_ret) + 1)
            cams = rng.choice(n_ret, k, replace=False)
            rbs.append([int(perm[n_ret + e])] + [int(perm[c]) for c in cams])
    if with_retained_rows:
        for _ in range(n_ret):
            k = rng.integers(1, 3)
            rbs.append([int(perm[c]) for c in rng.choice(n_ret, k, replace=False)])
    order = rng.permutation(len(rbs))
    return bs, el, [rbs[i] for i in order]


@pytest.mark.parametrize("seed", range(6))
def test_random_descriptions(bls, seed):
    rng = np.random.default_rng(100 + seed)
    bs, el, rbs = _random_description(rng, int(rng.integers(2, 12)), int(rng.integers(1, 40)), 3, seed % 2 == 0)
    for nchunks in (1, 5):
        st = bls.SchurStructure(bs, rbs, eliminated=el, nchunks=nchunks)
        ost = orc.Structure.from_description(bs, rbs, el, nchunks=nchunks)
        _same_structure(st, ost)
        _same_workspace(st, ost, nchunks)
        extra = [(int(a), int(b)) for a, b in rng.integers(0, st.nrblocks, (3, 2))]
        _same_pattern(bls, st, ost, extra)


@pytest.mark.parametrize("name", ["dense_50x2000", "sparse_1000x200k", "qr_500x100k", "batched_256", "pcg_10000x1M"])
def test_scene_layouts(bls, name):
    """Scaled-down scenes of every workload family: product layout == oracle layout."""
    spec = bls.scenes.scaled_down(bls.scenes.workload(name), ncams=40, npoints=600)
    sc = bls.scenes.Scene(spec)
    bs, el, ptr, idx = sc.description()
    st = bls.SchurStructure(bs, (ptr, idx), eliminated=el, nchunks=4)
    ost = orc.Structure.from_description(bs, (ptr, idx), el, nchunks=4)
    _same_structure(st, ost)
    _same_workspace(st, ost, 4)
    _same_pattern(bls, st, ost)


def test_rejected_descriptions(bls):
    for c in KA["rejected"]:
        el = c.get("el", [False, True, True])
        with pytest.raises(bls.ArgumentError) as ei:
            bls.SchurStructure(c["bs"], c["rbs"], eliminated=el)
        assert str(ei.value) == c["msg"]
    # an eliminated block in no row block is allowed on the Hessian path
    assert bls.SchurStructure([6, 3, 3], [[0, 1]], eliminated=[False, True, True]).nblocks() == 3
    with pytest.raises(bls.DimensionMismatch):
        bls.SchurStructure([6, 3, 3], [[0, 1]], eliminated=[False, True])
    with pytest.raises(bls.ArgumentError):
        bls.SchurStructure.positional([6, 6], [3, 3], [[0, 1, 0], [1]])
    with pytest.raises(bls.ArgumentError):
        bls.SchurStructure.positional([6, 6], [3, 3], [[0, 1], [1]], nchunks=0)
    st = bls.SchurStructure.positional([6, 6, 6, 6], [3] * 4, [[0, 1], [0, 1], [2, 3], [2, 3]])
    with pytest.raises(bls.ArgumentError):
        bls.build_schur_pattern(st, [(0, 4)])


@pytest.mark.parametrize("fx", [STANDARD, COUPLED_GROUPS], ids=["standard", "coupled_groups"])
def test_scalar_and_block_r_to_s_maps_agree(bls, fx):
    """build_r_to_s_map: the scalar-level form (R's block storage against the scalar CSC of S) equals the block-level
    one (test/schur_problems.jl:241-262); mapped slots are unique and in S's upper triangle; the count is every
    upper-triangle entry of the diagonal blocks plus every entry of the off-diagonal blocks
    (test/dampedlinearsolve_schurhessian.jl:108-114); the oracle's restatement agrees; and R's couplings without a slot
    in S are rejected."""
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    extra = fx.get("rr_pairs", ())
    pat = bls.build_schur_pattern(st, extra)
    R = bls.BlockSystem.retained(st, pat)
    pairs = bls.retained_block_pairs(R)
    assert {(max(a, b), min(a, b)) for a, b in extra} <= set(pairs)   # R's couplings are among its off-diagonal blocks
    # the retained pairs build the same pattern (they are the pattern's off-diagonal blocks)
    pat2 = bls.build_schur_pattern(st, pairs)
    np.testing.assert_array_equal(pat2.S_colptr, pat.S_colptr)
    np.testing.assert_array_equal(pat2.S_rowval, pat.S_rowval)
    m_block = bls.build_r_to_s_map(st, pat)
    m_scalar = bls.build_r_to_s_map_blocks(R, pat.S_colptr, pat.S_rowval, st.boffsets_r, pat.R_length)
    np.testing.assert_array_equal(m_block, m_scalar)
    o = orc.r_to_s_map_blocks_csc(st.r_dims, pat.block_colptr, pat.block_rowval, pat.R_block_start, pat.R_length, pat.S_colptr,
                                  pat.S_rowval, st.boffsets_r)
    np.testing.assert_array_equal(o, m_scalar)
    mapped = m_block[m_block >= 0]
    assert len(np.unique(mapped)) == len(mapped)
    cols = np.repeat(np.arange(st.nr), np.diff(pat.S_colptr))
    assert np.all(pat.S_rowval[mapped] <= cols[mapped])
    d = np.asarray(st.r_dims)
    expect = int(np.sum(d * (d + 1) // 2)) + sum(int(d[a] * d[b]) for a, b in pairs)
    assert len(mapped) == expect
    if extra:
        plain = bls.build_schur_pattern(st)
        with pytest.raises(bls.ArgumentError, match="is not present in the sparsity pattern of S"):
            bls.build_r_to_s_map_blocks(R, plain.S_colptr, plain.S_rowval, st.boffsets_r, pat.R_length)
        with pytest.raises(orc.OracleError, match="is not present in the sparsity pattern of S"):
            orc.r_to_s_map_blocks_csc(st.r_dims, pat.block_colptr, pat.block_rowval, pat.R_block_start, pat.R_length, plain.S_colptr,
                                      plain.S_rowval, st.boffsets_r)


def test_retained_block_pairs_known_answer(bls):
    """retained_block_pairs(H.R) contains the coupled-groups problem's retained-retained couplings
    (test/dampedlinearsolve_schurhessian.jl:108: (3, 1) and (4, 2), 1-based)."""
    fx = COUPLED_GROUPS
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    pat = bls.build_schur_pattern(st, fx.get("rr_pairs", ()))
    pairs = set(bls.retained_block_pairs(bls.BlockSystem.retained(st, pat)))
    assert {(2, 0), (3, 1)} <= pairs
    assert pairs == set(orc.retained_block_pairs(pat.block_colptr, pat.block_rowval))


def test_scalar_csc_r_to_s_map(bls):
    """build_r_to_s_map(R_sparse, S_sparse): positions found by binary search equal a linear search of S's column (the
    reference's own check, test/schur.jl:320-333, 488-489); an entry absent from S is rejected with its position."""
    fx = STANDARD
    st = bls.SchurStructure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    pat = bls.build_schur_pattern(st)
    rng = np.random.default_rng(4)
    n = st.nr
    # R: a random subset of S's stored entries, rows ascending in each column
    rc, rr = [0], []
    for j in range(n):
        rows = pat.S_rowval[pat.S_colptr[j]:pat.S_colptr[j + 1]]
        keep = rows[rng.random(len(rows)) < 0.6]
        rr.extend(keep.tolist())
        rc.append(len(rr))
    rc, rr = np.array(rc), np.array(rr, np.int64)
    expect = []
    for j in range(n):
        for k in range(rc[j], rc[j + 1]):
            lo, hi = pat.S_colptr[j], pat.S_colptr[j + 1]
            expect.append(lo + int(np.flatnonzero(pat.S_rowval[lo:hi] == rr[k])[0]))
    got = bls.build_r_to_s_map_scalar(rc, rr, pat.S_colptr, pat.S_rowval)
    np.testing.assert_array_equal(got, expect)
    np.testing.assert_array_equal(orc.r_to_s_map_csc(rc, rr, pat.S_colptr, pat.S_rowval), expect)
    # an entry of R outside S's pattern: S stores the upper block triangle, so column 0 holds no row of a later block
    j = 0
    missing = next(i for i in range(n) if i not in set(pat.S_rowval[pat.S_colptr[j]:pat.S_colptr[j + 1]].tolist()))
    rr2 = np.concatenate([np.sort(np.append(rr[:rc[1]], missing)), rr[rc[1]:]])
    rc2 = rc.copy()
    rc2[1:] += 1
    with pytest.raises(bls.ArgumentError, match=f"R entry \\({missing + 1}, {j + 1}\\) is not present"):
        bls.build_r_to_s_map_scalar(rc2, rr2, pat.S_colptr, pat.S_rowval)
    with pytest.raises(orc.OracleError, match=f"R entry \\({missing + 1}, {j + 1}\\) is not present"):
        orc.r_to_s_map_csc(rc2, rr2, pat.S_colptr, pat.S_rowval)
