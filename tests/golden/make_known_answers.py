"""Write known_answers.json: the literal expected results of BlockLinearSystems.jl's own tests for the layout path,
transcribed (0-based) from the cited test lines. The reference stores no golden value vectors (its tests draw random
values from Julia's Xoshiro), so these integer known answers are what pins the oracle's layout to the reference.

    python tests/golden/make_known_answers.py
"""
import json
from pathlib import Path

CASES = {
    # src/schur_structure.jl:43-47 (doctest): blockorder, nretained, blocksizes
    "doctest_structure": {
        "blocksizes": [3, 6, 3, 6], "rowblocks": [[0, 1], [1, 2], [2, 3], [1, 3]], "eliminated": [True, False, True, False],
        "blockorder": [1, 3, 0, 2], "nretained": 2, "layout_blocksizes": [6, 6, 3, 3],
    },
    # src/schur_description.jl:129-134 (doctest): SchurJacobianStructure blockorder, nretained, nblocks
    "doctest_jacobian_structure": {
        "blocksizes": [3, 6, 3, 6], "rowblocks": [[0, 1], [0, 3], [1, 2], [2, 3], [1]], "rowblocksizes": [2, 2, 2, 2, 6],
        "eliminated": [True, False, True, False], "blockorder": [1, 3, 0, 2], "nretained": 2, "nblocks": 4,
    },
    # test/schur.jl:459-463: expand_block_perm([2, 1, 3], [3, 2, 4]) == [4, 5, 1, 2, 3, 6, 7, 8, 9]
    "expand_block_perm": {"perm": [1, 0, 2], "sizes": [3, 2, 4], "expected": [3, 4, 0, 1, 2, 5, 6, 7, 8]},
    # test/schur.jl:465-475: sort_schur_blocks(Bool[0,1,0,1,1], [6,3,3,1,3], [[],[2,1],[],[1],[3,2]]) == [1,3,2,5,4]
    "sort_schur_blocks": {"is_elim": [False, True, False, True, True], "sizes": [6, 3, 3, 1, 3],
                          "couplings": [[], [1, 0], [], [0], [2, 1]], "expected": [0, 2, 1, 4, 3]},
    # test/schur_problems.jl:266-272: extra pairs add exactly two blocks to the coupled-groups pattern
    "coupled_groups_extra": {"extra": [[2, 0], [1, 3]], "added_blocks": 2},
    # test/schur_problems.jl:281-285: r->s map of the coupled-groups system with its retained pairs maps
    # 4*21 + 36*npairs entries (npairs = number of off-diagonal retained pairs of R)
    "coupled_groups_r_to_s_count": {"diag_upper_per_block": 21, "offdiag_per_block": 36},
    # test/qr_reduction.jl:176-178: bytes of SchurJacobianStructure(fill(6,10), fill(3,1000), [1:10 for each], fill(40,1000))
    "qr_bytes": {"nret": 10, "nelim": 1000, "rows": 40, "expected_bytes": 2 * 8 * 1000 * 43 * 64},
    # test/schur_description.jl:85-87: a row block touching no column block makes its own free group
    "qr_free_group": {"blocksizes": [6, 3, 3], "eliminated": [False, True, True], "rowblocks": [[0, 1], [], [2, 0]],
                      "rowblocksizes": [2, 1, 3], "ntables": 3, "free_rows": [1]},
    # test/kernels.jl:5-7: [1 1; 1 1+1e-6] is singular in Float32 and not in Float64 (undamped)
    "inv_sym_2x2": {"H": [[1.0, 1.0], [1.0, 1.000001]], "f32_success": False, "f64_success": True},
    # test/kernels.jl:19-24: not positive definite though the determinant is positive
    "inv_sym_not_pd": {"cases": [[[-2.0, 0.0], [0.0, -2.0]], [[-2.0, 0, 0], [0, -2.0, 0], [0, 0, 2.0]],
                                 [[1.0, 2, 0], [2, 1.0, 0], [0, 0, -1.0]], [[-1.0]], [[-1.0, 0], [0, -1.0]],
                                 [[-1.0, 0, 0], [0, -1.0, 0], [0, 0, -1.0]]]},
    # test/schur_description.jl:70-82: rejected descriptions and their messages (bs = [6,3,3], el = [F,T,T])
    "rejected": [
        {"bs": [6, 0, 3], "rbs": [[0, 1], [2, 0]], "msg": "Block 2 has dimension 0; dimensions must be between 1 and 65535"},
        {"bs": [6, 3, 65536], "rbs": [[0, 1], [2, 0]], "msg": "Block 3 has dimension 65536; dimensions must be between 1 and 65535"},
        {"bs": [6, 3, 3], "rbs": [[0, 1], [3]], "msg": "Row block 2 touches column block 4, but there are 3 column blocks"},
        {"bs": [6, 3, 3], "rbs": [[0, 1], [-1, 0]], "msg": "Row block 2 touches column block 0, but there are 3 column blocks"},
        {"bs": [6, 3, 3], "rbs": [[0, 1, 0], [2]], "msg": "Row block 1 lists column block 1 more than once"},
        {"bs": [6, 3, 3], "rbs": [[0, 1], [2, 0, 1]], "msg": "Row block 2 touches two eliminated column blocks, 3 and 2; a row block may touch at most one"},
        {"bs": [6, 3, 3], "rbs": [[0, 1], [2, 0]], "el": [True, True, True], "msg": "An elimination needs at least one retained and one eliminated column block; got 0 retained and 3 eliminated"},
        {"bs": [6, 3, 3], "rbs": [[0, 1], [2, 0]], "el": [False, False, False], "msg": "An elimination needs at least one retained and one eliminated column block; got 3 retained and 0 eliminated"},
    ],
}

if __name__ == "__main__":
    out = Path(__file__).with_name("known_answers.json")
    out.write_text(json.dumps(CASES, indent=1) + "\n")
    print(out)
