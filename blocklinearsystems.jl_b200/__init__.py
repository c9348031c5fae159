"""blsgpu: a B200 (sm_100a) implementation of BlockLinearSystems.jl's elimination path behind a C ABI.

The package directory is named `blocklinearsystems.jl_b200`; load it under the module name `blsgpu` with
`load_package()` in __graft_entry__.py (or any importlib loader), as the directory name is not an identifier.

Layout (host, integer):  SchurStructure, build_schur_pattern, build_r_to_s_map (block and scalar forms),
                         retained_block_pairs, sparse_with_map, BlockSystem
Device reduction:        SchurReductionWorkspace, reset_schur_sparse / reset_schur_dense,
                         reduce_schur_sparse / reduce_schur_dense, backsubstitute, scatter_copy,
                         symmetrifyfull / symmetrifyfull_
QR elimination:          SchurJacobianStructure, SchurBlockJacobian, QRReductionWorkspace, reduce_qr, qr_backsubstitute,
                         reduced_normal_sparse / reduced_normal_dense, reduced_diagonal_blocks, free_block_pairs,
                         reduced_residual, reduced_jacobian / reduced_jacobian_sparse, build_reduced_jacobian_pattern,
                         reduced_mul / reduced_tmul, lsmr_reduced (the matrix-free LSMR solve of the reduced problem),
                         qr_refine (iterative refinement of the QR route's solve against the FP64 normal equations)
Reduced solve:           BlockJacobi, factor_diagonal_blocks, solve_diagonal_blocks, PCGWorkspace (block-Jacobi PCG)
Learned preconditioner:  gnn.LearnedPreconditioner, gnn.train, gnn.init_params
Batches:                 batch.BatchedReduction (uneven problems as one plan, one CUDA graph)
Workloads:               scenes.workload, scenes.hessian_problem, scenes.jacobian_problem
"""
from ._lib import ArgumentError, BlsError, DimensionMismatch
from .layout import (DEFAULT_MIN_WORK, BlockSystem, SchurPattern, SchurStructure, build_r_to_s_map, build_r_to_s_map_blocks,
                     build_r_to_s_map_scalar, build_schur_pattern, retained_block_pairs, sparse_with_map)
from .reduction import (SchurReductionWorkspace, backsubstitute, context, reduce_schur_dense, reduce_schur_sparse,
                        prepare_scale, reset_reduce_schur_sparse_host, reset_schur_dense, reset_schur_sparse, scatter_copy,
                        symmetrifyfull, symmetrifyfull_)
from .qr import (QRReductionWorkspace, SchurBlockJacobian, assemble_hessian, jtj_diag, jtj_quadform, jtr, SchurJacobianStructure, free_block_pairs, qr_backsubstitute, reduce_qr,
                 reduced_diagonal_blocks, reduced_nrows, reduced_normal_dense, reduced_normal_sparse, reduced_residual,
                 reduced_jacobian, reduced_jacobian_sparse, build_reduced_jacobian_pattern, reduced_mul, reduced_tmul,
                 lsmr_reduced, LsmrResult, qr_refine, RefineResult)
from .pcg import BlockJacobi, PCGResult, PCGWorkspace, RefinedResult, factor_diagonal_blocks, solve_diagonal_blocks
from .dense import DenseCholesky
from . import batch, gnn, scenes

__all__ = [
    "ArgumentError", "BlsError", "DimensionMismatch", "DEFAULT_MIN_WORK", "BlockSystem", "SchurPattern",
    "build_r_to_s_map_blocks", "build_r_to_s_map_scalar", "retained_block_pairs", "SchurStructure", "build_r_to_s_map",
    "build_schur_pattern", "sparse_with_map", "SchurReductionWorkspace", "backsubstitute", "context", "reduce_schur_dense",
    "reduce_schur_sparse", "reset_reduce_schur_sparse_host", "reset_schur_dense", "reset_schur_sparse", "scatter_copy", "scenes", "QRReductionWorkspace",
    "SchurBlockJacobian", "SchurJacobianStructure", "assemble_hessian", "jtj_diag", "jtj_quadform", "jtr", "prepare_scale", "free_block_pairs", "qr_backsubstitute", "reduce_qr", "reduced_diagonal_blocks",
    "reduced_nrows", "reduced_normal_dense", "reduced_normal_sparse", "reduced_residual", "reduced_jacobian",
    "reduced_jacobian_sparse", "build_reduced_jacobian_pattern", "reduced_mul", "reduced_tmul", "lsmr_reduced", "LsmrResult", "qr_refine", "RefineResult", "BlockJacobi", "PCGResult", "PCGWorkspace", "RefinedResult", "DenseCholesky",
    "factor_diagonal_blocks", "solve_diagonal_blocks", "gnn", "batch", "symmetrifyfull", "symmetrifyfull_",
]
