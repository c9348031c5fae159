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
