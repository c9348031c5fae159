"""symmetrifyfull / symmetrifyfull! (src/SparseBlockLinearSystem.jl:288-341): the oracle pinned on the reference's own
known answers (test/SparseBlockLinearSystem.jl:140-210: the 6 x 6 system of block sizes [2, 3, 1] with blocks (2, 1),
(2, 2), (3, 2), (3, 3), its block subsets in any order, a boolean mask, the empty subset and the three errors), and on a
Schur pattern's retained storage against the densified symmetric CSC of makesparseindices (the reference's other
symmetrification); then the device (through the C ABI) bit-exact against the oracle, errors raised before any write."""
import numpy as np
import pytest
import torch

import oracle as orc
from fixtures import COUPLED_GROUPS, GAUGE, SCHUR_JL, STANDARD

# The reference test's system: block sizes [2, 3, 1]; indicestransposed over block rows r: r = 2 holds blocks (2, 1)
# and (2, 2), r = 3 holds (3, 2) and (3, 3) (0-based below); the data in constructor order.
BS = np.array([2, 3, 1])
IT_COLPTR = np.array([0, 0, 2, 4])
IT_ROWVAL = np.array([0, 1, 1, 2])
IT_STARTS = np.array([0, 6, 15, 18])
DATA = np.array([1, 2, 3, 4, 5, 6,            # block(bs, 2, 1) .= reshape(1:6, (3, 2))
                 7, 8, 9, 8, 10, 11, 9, 11, 12,   # block(bs, 2, 2) .= [7 8 9; 8 10 11; 9 11 12]
                 13, 14, 15,                 # block(bs, 3, 2) .= [13 14 15]
                 16], np.float64)            # block(bs, 3, 3) .= 16
OUT2 = np.array([[0, 0, 0, 0, 0, 0],
                 [0, 0, 0, 0, 0, 0],
                 [1, 4, 7, 8, 9, 0],
                 [2, 5, 8, 10, 11, 0],
                 [3, 6, 9, 11, 12, 0],
                 [0, 0, 13, 14, 15, 16]], np.float64)
OUTSYM = np.maximum(OUT2, OUT2.T)
SCALAR = (np.arange(0, 2), np.arange(2, 5), np.arange(5, 6))   # the scalar indices of blocks 1, 2, 3
ORDERS = ([2, 0], [1, 0], [2, 1, 0], [1, 2, 0], [0, 2])       # the reference's orders, 0-based


def sym(blocks=None, m=None, data=DATA):
    return orc.symmetrify_full(BS, IT_COLPTR, IT_ROWVAL, IT_STARTS, data, blocks, m)


def test_oracle_known_answers():
    np.testing.assert_array_equal(sym(), OUTSYM)
    np.testing.assert_array_equal(sym([1, 2]), OUTSYM[2:6, 2:6])
    np.testing.assert_array_equal(sym([0]), OUTSYM[0:2, 0:2])
    np.testing.assert_array_equal(sym(np.array([False, True, True])), OUTSYM[2:6, 2:6])
    assert sym([], 0).shape == (0, 0)
    for order in ORDERS:
        idx = np.concatenate([SCALAR[b] for b in order])
        np.testing.assert_array_equal(sym(order), OUTSYM[np.ix_(idx, idx)])


def test_oracle_errors():
    with pytest.raises(orc.OracleError, match="expected"):            # DimensionMismatch
        sym([1, 2], 3)
    with pytest.raises(orc.OracleError, match="BoundsError"):
        sym([9], 2)
    with pytest.raises(orc.OracleError, match="Block 2 is listed more than once"):
        sym([1, 2, 1], 7)
    with pytest.raises(orc.OracleError, match="Block 1 is listed more than once"):
        sym([0, 0], 4)


def test_oracle_later_of_two_mirrored_blocks_wins():
    """Blocks (2, 1) and (1, 2) both present: the reference's loop writes (2, 1) (block row 2) last."""
    cp, rv, st = np.array([0, 1, 2]), np.array([1, 0]), np.array([0, 2])
    data = np.array([1.0, 2.0, 3.0, 4.0])   # block (1, 2) = [1 2], block (2, 1) = [3; 4] (sizes [1, 2])
    out = orc.symmetrify_full([1, 2], cp, rv, st, data)
    np.testing.assert_array_equal(out, [[0, 3, 4], [3, 0, 0], [4, 0, 0]])


@pytest.mark.parametrize("fx", [SCHUR_JL, STANDARD, COUPLED_GROUPS, GAUGE], ids=["schur_jl", "standard", "coupled_groups", "gauge"])
def test_oracle_on_a_schur_pattern_matches_the_symmetric_csc(fx):
    ost = orc.Structure.positional(fx["r_dims"], fx["e_dims"], fx["couplings"])
    q = orc.Pattern(ost, fx.get("rr_pairs", ()))
    data = np.random.default_rng(7).standard_normal(q.R_length)
    full = orc.symmetrify_full(ost.r_dims, q.block_colptr, q.block_rowval, q.R_block_start, data)
    colptr, rowval, smap = q.sparse_indices(True)
    n = ost.nr
    dense = np.zeros((n, n))
    for j in range(n):
        dense[rowval[colptr[j]:colptr[j + 1]], j] = data[smap[colptr[j]:colptr[j + 1]]]
    np.testing.assert_array_equal(full, dense)
    # a subset in reverse order: the permuted principal submatrix
    starts = np.concatenate([[0], np.cumsum(ost.r_dims)])
    order = list(range(len(ost.r_dims)))[::-2]
    idx = np.concatenate([np.arange(starts[b], starts[b + 1]) for b in order])
    np.testing.assert_array_equal(orc.symmetrify_full(ost.r_dims, q.block_colptr, q.block_rowval, q.R_block_start, data, order),
                                  full[np.ix_(idx, idx)])


# ----- the device, through the C ABI -----

def _bsys(bls):
    return bls.BlockSystem(BS, IT_COLPTR, IT_ROWVAL, IT_STARTS)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_device_known_answers(bls, dtype):
    d = torch.from_numpy(DATA).to("cuda", dtype)
    b = _bsys(bls)
    assert np.array_equal(bls.symmetrifyfull(b, d).cpu().double().numpy(), OUTSYM)
    assert np.array_equal(bls.symmetrifyfull(b, d, [1, 2]).cpu().double().numpy(), OUTSYM[2:6, 2:6])
    assert np.array_equal(bls.symmetrifyfull(b, d, [0]).cpu().double().numpy(), OUTSYM[0:2, 0:2])
    assert np.array_equal(bls.symmetrifyfull(b, d, np.array([False, True, True])).cpu().double().numpy(), OUTSYM[2:6, 2:6])
    assert bls.symmetrifyfull(b, d, []).shape == (0, 0)
    for order in ORDERS:
        idx = np.concatenate([SCALAR[k] for k in order])
        assert np.array_equal(bls.symmetrifyfull(b, d, order).cpu().double().numpy(), OUTSYM[np.ix_(idx, idx)])


@pytest.mark.gpu
def test_device_errors_before_any_write(bls):
    d = torch.from_numpy(DATA).to("cuda")
    b = _bsys(bls)
    for blocks, m, err, msg in [([1, 2], 3, bls.DimensionMismatch, "expected"), ([9], 2, bls.ArgumentError, "BoundsError"),
                                ([1, 2, 1], 7, bls.ArgumentError, "Block 2 is listed more than once"),
                                ([0, 0], 4, bls.ArgumentError, "Block 1 is listed more than once")]:
        mat = torch.full((m, m), -7.0, dtype=torch.float64, device="cuda")
        with pytest.raises(err, match=msg):
            bls.symmetrifyfull_(mat, b, d, blocks)
        assert bool((mat == -7.0).all()), blocks


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_device_on_scene_retained_storage(bls, dtype):
    spec = bls.scenes.scaled_down(bls.scenes.workload("sparse_1000x200k"), ncams=60, npoints=900)
    p = bls.scenes.hessian_problem(spec)
    st, pat = p.structure, p.pattern
    data = p.R.astype(np.float32 if dtype == torch.float32 else np.float64)
    b = bls.BlockSystem.retained(st, pat)
    d = torch.from_numpy(data).to("cuda")
    ref = orc.symmetrify_full(st.r_dims, pat.block_colptr, pat.block_rowval, pat.R_block_start, data.astype(np.float64))
    assert np.array_equal(bls.symmetrifyfull(b, d).cpu().double().numpy(), ref)
    order = np.random.default_rng(3).permutation(st.nrblocks)[:25]
    sub = orc.symmetrify_full(st.r_dims, pat.block_colptr, pat.block_rowval, pat.R_block_start, data.astype(np.float64), order)
    assert np.array_equal(bls.symmetrifyfull(b, d, order).cpu().double().numpy(), sub)
