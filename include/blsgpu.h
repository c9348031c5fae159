/*
 * blsgpu.h — C ABI of libblsgpu.so, the B200 (sm_100a) implementation of BlockLinearSystems.jl's elimination path.
 *
 * Conventions
 *   - Plain C types only. Integers are int64_t; every index and offset is 0-based (the Julia caller subtracts 1).
 *   - Arrays named *_dev are device pointers on the context's device; everything else is host memory.
 *   - `dtype` selects the element type T of the block storage (R, E, C, S, factored tables): BLS_F64 or BLS_F32.
 *     Gradients, right-hand sides, solutions, lambda, damping scalings and conditioning scales are always double,
 *     as in the reference (src/schur_linear_systems.jl:11-13, src/schur_reduction.jl:21, src/qr_reduction.jl:8-10).
 *     With BLS_F32 the kernels run the mixed form: FP32 storage and FP32 pair products and accumulation, with the
 *     damped point-block inverse, z = E^-1 b_e, the gradient and the QR column norms / reflector scaling in FP64.
 *   - Work runs on the context's stream. A call that takes a host `int64_t* failed_block` synchronises and returns the
 *     reduction's verdict; passing NULL makes the call asynchronous (read it later with the *_query_status call).
 *   - Device memory is allocated by the create calls (contexts, plans, solvers) and, once per plan, by the first call
 *     of bls_reduced_tmul and bls_lsmr_reduced (their scratch, kept in the plan); bls_symmetrify_full stages its block
 *     list in stream-ordered memory (cudaMallocAsync) for the call. Kernels otherwise use only the caller's buffers
 *     and the plan's own scratch; bls_reduce_schur_dense_noalloc allocates nothing.
 *
 * Status codes: BLS_OK, BLS_NOT_PD (the reference's `false`: a singular / non-finite eliminated block; the lowest
 * such block, 1-based as the reference's failed_block[], is reported), and negative errors. Argument errors are
 * reported before any output is written, as the reference throws before any work (src/utils.jl:100-107).
 */
#ifndef BLSGPU_H
#define BLSGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BLS_OK 0
#define BLS_NOT_PD 1          /* reduce_schur_*! / reduce_qr! returned false (src/schur_reduction.jl:233-257) */
#define BLS_NOT_CONVERGED 2   /* an iterative solve stopped at its iteration limit above its tolerance */
#define BLS_EINVAL (-1)       /* ArgumentError (bad lambda / scaling / structure) */
#define BLS_EDIM (-2)         /* DimensionMismatch */
#define BLS_EPATTERN (-3)     /* a block missing from the sparse pattern (throw_missing_block, src/utils.jl:109) */
#define BLS_ECUDA (-4)        /* a CUDA runtime error */
#define BLS_EUNSUPPORTED (-5) /* a size this build does not handle (see the call's comment) */
#define BLS_ENOMEM (-6)

#define BLS_F64 0
#define BLS_F32 1

typedef struct bls_ctx bls_ctx;
typedef struct bls_structure bls_structure;
typedef struct bls_pattern bls_pattern;
typedef struct bls_schur_plan bls_schur_plan;
typedef struct bls_qr_structure bls_qr_structure;
typedef struct bls_qr_plan bls_qr_plan;
typedef struct bls_pcg_plan bls_pcg_plan;
typedef struct bls_block_jacobi bls_block_jacobi;
typedef struct bls_gnn bls_gnn;

int bls_version(void);
/* Message of the last error on the calling thread. */
const char* bls_last_error(void);

/* ---------------------------------------------------------------------------------------------------------------
 * Context: one device, one stream.
 * ------------------------------------------------------------------------------------------------------------- */
int bls_ctx_create(int device, bls_ctx** out);
int bls_ctx_destroy(bls_ctx* ctx);
/* Run the context's work on `cuda_stream` (a cudaStream_t; NULL = the legacy default stream). */
int bls_ctx_set_stream(bls_ctx* ctx, void* cuda_stream);
int bls_ctx_synchronize(bls_ctx* ctx);

/* ---------------------------------------------------------------------------------------------------------------
 * Host-side layout (integer, bit-exact with the reference). A Julia caller already has these from its own
 * SchurStructure and may skip straight to bls_schur_plan_create; the Python mirror builds them here.
 * ------------------------------------------------------------------------------------------------------------- */

/* SchurStructure(blocksizes, rowblocks; eliminated, nchunks, min_work) (src/schur_description.jl:97-101,
 * describe_elimination :16-89, sort_schur_blocks src/schur_structure.jl:204-228, constructor :70-166).
 * rowblocks in CSR form: row block k touches column blocks rowblock_idx[rowblock_ptr[k] .. rowblock_ptr[k+1]). */
int bls_structure_from_description(int64_t nblocks, const int64_t* blocksizes, int64_t nrowblocks,
                                   const int64_t* rowblock_ptr, const int64_t* rowblock_idx, const uint8_t* eliminated,
                                   int64_t nchunks, int64_t min_work, bls_structure** out);
/* The positional constructor SchurStructure(r_dims, e_dims, couplings) (src/schur_structure.jl:70-166).
 * couplings in CSR form over the eliminated blocks, retained indices 0-based. */
int bls_structure_positional(int64_t nrblocks, const int64_t* r_dims, int64_t neblocks, const int64_t* e_dims,
                             const int64_t* coupling_ptr, const int64_t* coupling_idx, int64_t nchunks,
                             int64_t min_work, bls_structure** out);
/* Field getter: returns the field's length and copies it into `out` when `out` is not NULL; -1 for an unknown name.
 * Fields: nr nrblocks neblocks r_dims e_dims boffsets_r boffsets_e eoffsets eliminated_ptr entry_retained coffsets
 * max_coupled_dim order retained_pairs chunks retained_ptr retained_entry entry_eliminated col_chunks. */
int64_t bls_structure_field(const bls_structure* st, const char* name, int64_t* out);
int bls_structure_destroy(bls_structure* st);

/* build_schur_pattern(structure; extra_blocks) (src/schur_structure.jl:241-323). extra_pairs: nextra (i, j) pairs.
 * Fields: block_colptr block_rowval block_row_offsets col_heights S_colptr S_rowval diag_inds, and for the sparse
 * retained storage on that pattern (src/schur_hessian.jl:286): R_block_start R_length. */
int bls_schur_pattern_build(const bls_structure* st, int64_t nextra, const int64_t* extra_pairs, bls_pattern** out);
int64_t bls_pattern_field(const bls_pattern* p, const char* name, int64_t* out);
int bls_pattern_destroy(bls_pattern* p);
/* build_r_to_s_map(R, pattern, boffsets_r), block-level form (src/schur_structure.jl:406-431), for the retained
 * storage laid out on the pattern. out[R_length]; -1 marks an unmapped entry (the reference's 0). */
int bls_build_r_to_s_map(const bls_structure* st, const bls_pattern* p, int64_t* out);
/* The scalar-level forms of build_r_to_s_map, against a scalar CSC pattern of S (S_colptr / S_rowval, 0-based, rows
 * sorted within each column; e.g. the pattern's S_colptr / S_rowval). Positions are found by binary search in S's
 * column; an entry absent from S is BLS_EINVAL with the reference's message (1-based indices).
 * bls_r_to_s_map_csc: build_r_to_s_map(R_sparse, S_sparse) (src/schur_structure.jl:336-353), R a CSC of ncols
 *   columns: out[nnz(R)] = the position in S.nzval of each stored entry of R.
 * bls_r_to_s_map_blocks_csc: build_r_to_s_map(R_sys, S_sparse, boffsets_r) (src/schur_structure.jl:363-397), R_sys a
 *   block-square SparseBlockLinearSystem given by its nb block sizes and indicestransposed (a CSC over block rows r:
 *   block (r, it_rowval[k]) starts at data[it_nzval[k]], column-major), boffsets_r[nb] the blocks' first scalar
 *   rows: out[data_len], a diagonal block's upper triangle and every entry of a block below the diagonal (placed in
 *   S's upper triangle), -1 elsewhere (the reference's 0). */
int bls_r_to_s_map_csc(int64_t ncols, const int64_t* R_colptr, const int64_t* R_rowval, const int64_t* S_colptr,
                       const int64_t* S_rowval, int64_t* out);
int bls_r_to_s_map_blocks_csc(int64_t nb, const int64_t* blocksizes, const int64_t* it_colptr, const int64_t* it_rowval,
                              const int64_t* it_nzval, int64_t data_len, const int64_t* S_colptr, const int64_t* S_rowval,
                              const int64_t* boffsets_r, int64_t* out);
/* makesparseindices / sparse_with_map (src/SparseBlockLinearSystem.jl:233-282, 343-354) for that retained storage:
 * the CSC pattern (colptr[nr+1], rowval[nnz]) and the integer scatter map[nnz] (0-based positions in the storage).
 * Returns nnz (pass NULL outputs to query it), or a negative status. */
int64_t bls_sparse_indices(const bls_structure* st, const bls_pattern* p, int symmetric, int64_t* colptr,
                           int64_t* rowval, int64_t* map);

/* ---------------------------------------------------------------------------------------------------------------
 * Device plan of a Schur elimination: the structure and pattern uploaded once, plus the plan's scratch (the
 * E_inv / z caches of SchurReductionWorkspace, src/schur_reduction.jl:16-27, and a status word).
 * ------------------------------------------------------------------------------------------------------------- */
typedef struct bls_schur_plan_desc {
  int64_t nrblocks, neblocks;
  const int64_t* r_dims;          /* [nrblocks] */
  const int64_t* e_dims;          /* [neblocks]; 1..3 supported on the device */
  const int64_t* eliminated_ptr;  /* [neblocks+1] point-major CSR of the couplings */
  const int64_t* entry_retained;  /* [ncouplings] ascending within each eliminated block */
  const int64_t* coffsets;        /* [ncouplings] start of each d_e x d_r coupling block in C_data */
  const int64_t* eoffsets;        /* [neblocks]  start of each d_e x d_e block in E_data */
  /* sparse pattern (may be NULL for a dense-only plan) */
  const int64_t* block_colptr;      /* [nrblocks+1] */
  const int64_t* block_rowval;      /* [nblocks_S] */
  const int64_t* block_row_offsets; /* [nblocks_S] */
  const int64_t* col_heights;       /* [nrblocks] */
  const int64_t* S_colptr;          /* [nr+1] */
  const int64_t* S_rowval;          /* [nnz_S] (needed only for conditioning scales) */
  const int64_t* diag_inds;         /* [nr] */
  const int64_t* r_to_s_map;        /* [R_length], -1 = unmapped */
  int64_t R_length;
} bls_schur_plan_desc;

/* The device plan of a Schur reduction (the reference's SchurReductionWorkspace plus the pattern). Retained blocks of 1
 * to 16 variables, eliminated blocks of 1 to 16 (closed-form inverse up to 3, Cholesky above; BLS_EUNSUPPORTED
 * beyond); uniform 6 / 3 blocks in the canonical layout take the fast kernels. */
int bls_schur_plan_create(bls_ctx* ctx, const bls_schur_plan_desc* desc, bls_schur_plan** out);
int bls_schur_plan_destroy(bls_schur_plan* plan);
/* Device bytes the plan holds (index arrays + scratch). */
int64_t bls_schur_plan_device_bytes(const bls_schur_plan* plan);

/* reset_schur_sparse!(nzval, R_nzval, r_to_s_map, diag_inds, scaling_r, lambda, ws, s_r)
 * (src/schur_reduction.jl:416-436): S = R + lambda*diag(scaling_r) (scaled by s_r when given), failure word reset.
 * scaling_r_dev[nr]; s_r_dev may be NULL (UnitScale). */
int bls_reset_schur_sparse(bls_schur_plan* plan, int dtype, void* S_nzval_dev, const void* R_data_dev,
                           const double* scaling_r_dev, double lambda, const double* s_r_dev);
/* reset_schur_dense!(S, R, scaling_r, lambda, ws, s_r) (src/schur_reduction.jl:389-407); S and R column-major nr x nr. */
int bls_reset_schur_dense(bls_schur_plan* plan, int dtype, void* S_dev, const void* R_dev,
                          const double* scaling_r_dev, double lambda, const double* s_r_dev);

/* reduce_schur_sparse!(S, g_S, b_r, b_e, scaling_e, lambda, structure, E_data, C_data, block_colptr, block_rowval,
 * block_row_offsets, col_heights, ws, s_r, s_e) (src/schur_reduction.jl:489-507): S.nzval -= C' E^-1 C over every
 * eliminated block, g_S = s_r.*b_r - C' E^-1 b_e. S_nzval must hold the reset system. Returns BLS_OK, BLS_NOT_PD
 * (failed_block = lowest failing eliminated block, 1-based; S and g_S then untouched) or an error.
 * failed_block NULL: asynchronous, query with bls_schur_query_status. */
int bls_reduce_schur_sparse(bls_schur_plan* plan, int dtype, void* S_nzval_dev, double* g_S_dev, const double* b_r_dev,
                            const double* b_e_dev, const double* scaling_e_dev, double lambda, const void* E_data_dev,
                            const void* C_data_dev, const double* s_r_dev, const double* s_e_dev,
                            int64_t* failed_block);
/* reduce_schur_dense!(S, g_S, b_r, b_e, scaling_e, lambda, structure, E_data, C_data, ws, s_r, s_e)
 * (src/schur_reduction.jl:465-479): the same into the upper triangle of a column-major nr x nr S. */
int bls_reduce_schur_dense(bls_schur_plan* plan, int dtype, void* S_dev, double* g_S_dev, const double* b_r_dev,
                           const double* b_e_dev, const double* scaling_e_dev, double lambda, const void* E_data_dev,
                           const void* C_data_dev, const double* s_r_dev, const double* s_e_dev,
                           int64_t* failed_block);
/* reset_schur_sparse!(S.nzval, R, r_to_s_map, diag_inds, scaling_r, lambda, ws) followed by reduce_schur_sparse!(S, g_S,
 * b_r, b_e, scaling_e, lambda, ...) (src/schur_reduction.jl:416-436 and 489-507) on HOST buffers: the pair of calls a
 * caller whose arrays live in host memory makes, with the host-to-device copies overlapped with the reduction. The
 * points are cut into 16 stages of about equal coupling count; R, the point data (E, b_e, scaling_e) and then C are
 * copied on a second stream, and each stage's pairs are reduced while the next stage's part of C is still being
 * copied. Outputs S_nzval[nnz] and g_S[nr] are written only on BLS_OK; on
 * BLS_NOT_PD (failed_block as above) or an error they are untouched. Page-locked host buffers give the overlap;
 * pageable ones work, with copies staged by the driver. Sparse plans on the d_r = 6 / d_e = 3 fast path whose
 * diag_inds lie in their own columns, no conditioning scales (BLS_EUNSUPPORTED otherwise). The device copies of the
 * inputs are allocated on the plan at the first call and freed with it. Synchronous. */
int bls_reset_reduce_schur_sparse_host(bls_schur_plan* plan, int dtype, void* S_nzval, double* g_S, const void* R_data,
                                       const double* scaling_r, double lambda, const double* b_r, const double* b_e,
                                       const double* scaling_e, const void* E_data, const void* C_data, int64_t* failed_block);
/* Instrumentation (no counterpart in the reference): with timing on, CUDA events bracket the pair kernel of every
 * reduction on the plan's stream. bls_schur_plan_counters synchronises on the last event, reports the device kernel
 * launches issued since the previous read, the summed pair-kernel time and its number of launches, and resets them. */
int bls_schur_plan_instrument(bls_schur_plan* plan, int timing);
/* Phase-2 kernel of the d_r = 6 / d_e = 3 fast path (no counterpart in the reference): 0 = block-column owned,
 * 1 = block owned, six lanes per pair list (the default), 2 = block owned, a lane per pair and a warp per pair list,
 * 3 = block-column owned with visits staged in chunks (sparse S without conditioning scales; otherwise as 1),
 * 4 = point-major, six lanes per pair, entries added into S with vector reductions (as 1 when S has 2^25 or more
 * blocks). All compute the same reduction; the choice is kept for comparisons and for autotuning. */
int bls_schur_plan_set_kernel(bls_schur_plan* plan, int which);
/* No counterpart in the reference (a tuning knob of this build's schedule): rebuild the column-owned schedule (which = 5)
 * with units of at most `unit` pairs for both storage types (1..4096; at plan creation 20 for FP32 storage and 16 for
 * FP64), a unit being one thread's run of one S block's
 * pairs between two writes to the column tile. Sparse plans on the 6/3 fast path only (BLS_EUNSUPPORTED otherwise);
 * on failure the previous schedule stays. Synchronises. */
int bls_schur_plan_set_stage_unit(bls_schur_plan* plan, int unit);
/* No counterpart in the reference (a batch of the reference's calls in one plan): declare that the plan's structure is
 * the disjoint union of `nprob` independent problems, problem p owning eliminated blocks [point_off[p],
 * point_off[p+1]), retained blocks [camera_off[p], camera_off[p+1]), rows [row_off[p], row_off[p+1]) of g_S and
 * entries [nnz_off[p], nnz_off[p+1]) of S.nzval (host arrays of nprob + 1, from 0 to the plan's sizes). Each problem
 * then fails on its own, as a separate reduce_schur_sparse! call would (src/schur_reduction.jl:233-257): a problem with
 * a failing eliminated block keeps its reset S and its g_S, the others are reduced; the reduction's own status is
 * BLS_OK and the problems' verdicts are read with bls_schur_plan_problem_status. Sparse plans on the 6/3 fast path
 * only; nprob = 0 removes the partition. */
int bls_schur_plan_set_problems(bls_schur_plan* plan, int64_t nprob, const int64_t* point_off, const int64_t* camera_off,
                                const int64_t* row_off, const int64_t* nnz_off);
/* Per problem of the last reduction: 0, or its lowest failing eliminated block (1-based, local to the problem) in
 * failed_blocks[nprob] (host). Returns BLS_NOT_PD if any problem failed. Synchronises. */
int bls_schur_plan_problem_status(bls_schur_plan* plan, int64_t* failed_blocks);
/* No counterpart in the reference (instrumentation): the name of the phase-2 kernel that the next reduction of storage
 * type `dtype` launches on this plan, for a dense (`dense` != 0) or sparse S, with conditioning scales (`scaled` != 0)
 * or without, written NUL-terminated into buf[cap]. */
int bls_schur_plan_phase2_kernel(bls_schur_plan* plan, int dtype, int dense, int scaled, char* buf, int64_t cap);
int bls_schur_plan_counters(bls_schur_plan* plan, int64_t* launches, double* pair_kernel_ms, int64_t* pair_kernel_launches);

/* Status of the last reduction on this plan (synchronises): BLS_OK / BLS_NOT_PD / BLS_EINVAL. */
int bls_schur_query_status(bls_schur_plan* plan, int64_t* failed_block);

/* dot(x, H, y) (schur_bilinear, src/linalg.jl:133-262) of a SchurBlockHessian with R on S's pattern (dense = 0:
 * S.nzval layout, its upper part; dense = 1: column-major nr x nr, upper triangle), E_data and C_data in the plan's
 * layout: *result = x'Hy in FP64 for x, y = [x_r; x_e] (synchronises). Sparse R needs S_rowval in the plan.
 * bls_hessian_diagonal: d[nr + ne] = [diag R; the diagonals of the E blocks] (the diagonal a conditioned Hessian system
 * hands prepare_scale!). */
int bls_hessian_bilinear(bls_schur_plan* plan, int dtype, const void* R_dev, int dense, const void* E_data_dev, const void* C_data_dev,
                         const double* x_dev, const double* y_dev, double* result);
int bls_hessian_diagonal(bls_schur_plan* plan, int dtype, const void* R_dev, int dense, const void* E_data_dev, double* d_dev);

/* The point term of the reduced operator in FP64 (no counterpart in the reference, which forms S instead):
 * y = y0 - sum over eliminated blocks of C' E^-1 C x, with E^-1 the FP64 inverse of the damped point block from the
 * plan's last successful reduction and C its coupling blocks (dtype storage, as reduced); y and y0 distinct. With y0 =
 * (R + lambda diag(scaling_r)) x it is the reduced matrix times x, formed exactly in FP64 from the stored blocks.
 * Unconditioned reductions, eliminated blocks of size <= 3. */
int bls_schur_apply_elimination(bls_schur_plan* plan, int dtype, double* y_dev, const double* y0_dev, const double* x_dev,
                                const void* C_data_dev);

/* backsubstitute!(x_e, x_r, structure, C_data, ws, s_r, s_e) (src/schur_reduction.jl:519-576):
 * x_e = z - E^-1 sum_r C_er x_r per eliminated block, from the caches of the last successful reduction. */
int bls_backsubstitute(bls_schur_plan* plan, int dtype, double* x_e_dev, const double* x_r_dev,
                       const void* C_data_dev, const double* s_r_dev, const double* s_e_dev);

/* No counterpart in the reference: reduce_schur_dense! for callers that cannot allocate device memory (a caller whose
 * device memory belongs to an allocator it does not own, such as CUDA.jl's pool or PyTorch's caching allocator, or
 * one held to a fixed memory budget). Every other reduction needs a plan, which allocates; this call takes the
 * structure's eliminated_ptr[neblocks+1] and entry_retained[ncouplings] (0-based) already in device memory and keeps
 * its scratch (each point's damped inverse and z, and a status word) in a static device array of the library, so it
 * allocates nothing. Scope: retained blocks of 6 and eliminated blocks of 3 in the canonical layout (coupling c at
 * C_data[18c], point e at E_data[9e]), dense column-major S (nr = 6 nrblocks) already holding the reset system, at most
 * BLS_NOALLOC_MAX_POINTS eliminated blocks (larger sizes: BLS_EUNSUPPORTED, nothing launched). Results are those of
 * bls_reduce_schur_dense. With a host `failed_block` the call synchronises on `cuda_stream` and returns the verdict:
 * BLS_NOT_PD with the lowest failing block (1-based), or BLS_EINVAL for a bad scaling_e entry or a malformed
 * structure (an eliminated_ptr or entry_retained index out of range, or entry_retained not ascending within a point),
 * in which case S and g_S are left untouched. With failed_block NULL the call only queues its kernels; the verdict
 * stays in the array's status words until the next call on the device and is read with
 * bls_reduce_schur_dense_noalloc_status. The array is shared by all calls on a device and keeps the last call's
 * contents; calls whose work overlaps on the GPU race on it. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and caches it: make that first call before any stream capture. */
#define BLS_NOALLOC_MAX_POINTS 65536
int bls_reduce_schur_dense_noalloc(void* cuda_stream, int dtype, int64_t nrblocks, int64_t neblocks, int64_t ncouplings,
                                   const int64_t* eliminated_ptr_dev, const int64_t* entry_retained_dev, void* S_dev,
                                   double* g_S_dev, const double* b_r_dev, const double* b_e_dev,
                                   const double* scaling_e_dev, double lambda, const void* E_dev, const void* C_dev,
                                   int64_t* failed_block);
/* No counterpart in the reference: the verdict of the last bls_reduce_schur_dense_noalloc call on the current device
 * (the same codes and failed_block as its synchronous form), read from the static array's status words after the work
 * queued on `cuda_stream`. Synchronises on `cuda_stream`; allocates nothing. */
int bls_reduce_schur_dense_noalloc_status(void* cuda_stream, int64_t* failed_block);

/* ---------------------------------------------------------------------------------------------------------------
 * QR elimination (src/schur_jacobian.jl, src/qr_reduction.jl, src/qr_reduced.jl). The Jacobian is stored as one table
 * per eliminated block (its rows, then d_e damping rows; columns: the coupled retained blocks' columns in ascending
 * order, then the d_e eliminated columns, column-major, `raw_offsets`), then one table per free group of row blocks
 * that touch no eliminated block; the residual is a separate double vector (`residual_offsets`).
 * ------------------------------------------------------------------------------------------------------------- */

/* SchurJacobianStructure(blocksizes, rowblocks, rowblocksizes; eliminated, nchunks, min_work)
 * (src/schur_description.jl:137-189), rowblocks in CSR form as for bls_structure_from_description. */
int bls_qr_structure_from_description(int64_t nblocks, const int64_t* blocksizes, int64_t nrowblocks, const int64_t* rowblock_ptr,
                                      const int64_t* rowblock_idx, const int64_t* rowblocksizes, const uint8_t* eliminated,
                                      int64_t nchunks, int64_t min_work, bls_qr_structure** out);
/* SchurJacobianStructure(structure, e_rows; free_rows, free_retained, nchunks) (src/schur_jacobian.jl:59-160):
 * e_rows[neblocks]; free group g has free_rows[g] rows and retained blocks free_idx[free_ptr[g] .. free_ptr[g+1]). */
int bls_qr_structure_positional(const bls_structure* st, const int64_t* e_rows, int64_t nfree, const int64_t* free_rows,
                                const int64_t* free_ptr, const int64_t* free_idx, int64_t nchunks, bls_qr_structure** out);
/* Fields (as bls_structure_field): ntables raw_length residual_length e_rows free_rows table_nrows table_ncols table_top
 * table_offsets raw_offsets residual_offsets reduced_offsets table_ptr entry_retained entry_col entry_table retained_ptr
 * retained_entry doffsets col_chunks row_table row_first row_nrows row_ptr row_blocks. */
int64_t bls_qr_structure_field(const bls_qr_structure* q, const char* name, int64_t* out);
/* build_reduced_jacobian_pattern (src/qr_reduced.jl:284-310): the CSC pattern of J~ (reduced_nrows x nr), 0-based:
 * column c of retained block r stores the reduced rows of every table coupled to r, tables in ascending order. Returns
 * nnz; fills colptr[nr + 1] and rowval[nnz] when they are not NULL. */
int64_t bls_reduced_jacobian_pattern(const bls_qr_structure* q, int64_t* colptr, int64_t* rowval);
/* The SchurStructure the QR structure is built on (a copy; destroy it with bls_structure_destroy). */
int bls_qr_structure_schur(const bls_qr_structure* q, bls_structure** out);
int bls_qr_structure_destroy(bls_qr_structure* q);

/* Device plan of a QR elimination (QRReductionWorkspace, src/qr_reduction.jl:11-24, plus the J~'J~ work lists).
 * d_r <= 16; an eliminated block's table (8 bytes per entry of its M x C columns plus its residual) must fit in
 * 224 KB of shared memory (BLS_EUNSUPPORTED otherwise). */
typedef struct bls_qr_plan_desc {
  int64_t nrblocks, neblocks, ntables;
  const int64_t* r_dims;            /* [nrblocks] */
  const int64_t* e_dims;            /* [neblocks] */
  const int64_t* table_nrows;       /* [ntables] */
  const int64_t* table_ncols;       /* [ntables] including the residual column */
  const int64_t* table_top;         /* [ntables] d_e, 0 for free tables */
  const int64_t* table_ptr;         /* [ntables+1] entries of each table */
  const int64_t* entry_retained;    /* [nentries] */
  const int64_t* entry_col;         /* [nentries] first column of the entry in its table */
  const int64_t* raw_offsets;       /* [ntables+1] */
  const int64_t* residual_offsets;  /* [ntables+1] */
  /* sparse pattern of J~'J~ (may be NULL for a dense-only plan), as in bls_schur_plan_desc */
  const int64_t* block_colptr;
  const int64_t* block_rowval;
  const int64_t* block_row_offsets;
  const int64_t* col_heights;
  const int64_t* S_colptr;
} bls_qr_plan_desc;

int bls_qr_plan_create(bls_ctx* ctx, const bls_qr_plan_desc* desc, bls_qr_plan** out);
int bls_qr_plan_destroy(bls_qr_plan* plan);
/* No counterpart in the reference (iterative refinement of the QR route, the reduced solve being mixed precision; the
 * reference solves once, src/qr_linear_systems.jl:250-300). The steps of one refinement step x += dx of the damped
 * least-squares problem min ||J x - r||^2 + lambda x' diag(scaling) x, x = [x_r; x_e] (nr + ne, FP64):
 *  - bls_qr_normal_residual: d = J' (r - J x) - lambda scaling .* x in FP64 from the RAW tables J (raw_offsets layout,
 *    storage type `dtype`; the damping rows of the eliminated tables are ignored, their damping is the lambda term) and
 *    the raw residual r; y (residual_length doubles) receives r - J x per row;
 *  - bls_qr_reduce_rhs: from the FACTORED tables F of the last reduce_qr, per eliminated block w = U^-T d_e (ne
 *    doubles) and d_r = d[0:nr] - sum B' w, so that (J~'J~ + lambda diag(scaling_r)) dx_r = d_r;
 *  - bls_qr_backsubstitute_rhs: dx_e = U^-1 (w - B dx_r).
 * The reduced solve between the last two is the caller's (bls_dense_cholesky_shifted + bls_dense_cholesky_solve, or a
 * PCG on the sparse J~'J~). */
int bls_qr_normal_residual(bls_qr_plan* plan, int dtype, const void* J_dev, const double* r_dev, const double* scaling_dev,
                           double lambda, const double* x_dev, double* y_dev, double* d_dev);
int bls_qr_reduce_rhs(bls_qr_plan* plan, int dtype, const void* F_dev, const double* d_dev, double* w_dev, double* d_r_dev);
int bls_qr_backsubstitute_rhs(bls_qr_plan* plan, int dtype, const void* F_dev, const double* w_dev, const double* x_r_dev,
                              double* x_e_dev);
/* No counterpart in the reference (a staging choice of this build): how the table kernels (reduce_qr, the Gram kernels
 * of reduced_normal_*, reduced_diagonal_blocks and bls_assemble_hessian) bring each table into shared memory. bulk != 0
 * (the default): one bulk (TMA) copy per contiguous span, completed on an mbarrier; 0: element-wise asynchronous copies.
 * Buffers whose starts are not 16-byte aligned are always staged element-wise. Results are identical either way. */
int bls_qr_plan_set_staging(bls_qr_plan* plan, int bulk);

/* reduce_qr!(ws, J, scaling_e, lambda, s) (src/qr_reduction.jl:162-187): every eliminated table copied from the raw
 * tables Rw / residual Rr into F / Fr, damped with sqrt(lambda*scaling_e) (times s_e) and QR-factored in place; free
 * tables copied. s_dev: conditioning scale over all the variables [s_r; s_e], or NULL. Returns BLS_OK, BLS_NOT_PD
 * (failed_block = the lowest eliminated block with a non-finite table or a numerically singular U, 1-based) or an error;
 * failed_block NULL = asynchronous. */
int bls_reduce_qr(bls_qr_plan* plan, int dtype, void* F_dev, double* Fr_dev, const void* Rw_dev, const double* Rr_dev,
                  const double* scaling_e_dev, double lambda, const double* s_dev, int64_t* failed_block);
/* The normal equations of the raw Jacobian in the Hessian layout of the same structure (no device counterpart in the
 * reference: its callers fill a SchurBlockHessian with addblock!, src/schur_assembly.jl:140-246, and its fixtures form
 * H = J'J, b = J'r in FP64, test/fixtures/QRFixtures.jl:109-120): over the data rows of every table (not the damping
 * rows), E_data (d_e x d_e per eliminated block, SchurStructure's eoffsets), C_data (d_e x d_r per coupling, its
 * coffsets), R = the retained blocks of J'J on the reduced pattern (dense = 0: S.nzval layout, upper triangle of the
 * diagonal blocks, other entries zero; dense = 1: column-major nr x nr, upper triangle) and b = J'r = [b_r; b_e]
 * (FP64). Sums accumulate in FP64; E and C are rounded once, R once per table. R on the pattern resets a Schur plan
 * built with the identity r -> s map. */
int bls_assemble_hessian(bls_qr_plan* plan, int dtype, const void* Rw_dev, const double* Rr_dev, void* E_data_dev,
                         void* C_data_dev, void* R_dev, int dense, double* b_dev);
/* Quantities of the full problem from tables D (the raw J.data or the factored ws.factored, dtype) and their FP64
 * residual Rv (J.r or ws.fres), over every row of each table, FP64 sums:
 * jtr!(g, src) (src/qr_reduced.jl:575-584): g[nr + ne] = J'r, retained columns summed per block, then each point's;
 * jtj_diag!(d, src) (:586-595): d[nr + ne] = the squared column norms of J;
 * jtj_quadform(src, v) (:597-640): *result = ||J v||^2 for v[nr + ne] (synchronises). */
int bls_jtr(bls_qr_plan* plan, int dtype, double* g_dev, const void* D_dev, const double* Rv_dev);
int bls_jtj_diag(bls_qr_plan* plan, int dtype, double* d_dev, const void* D_dev);
int bls_jtj_quadform(bls_qr_plan* plan, int dtype, const void* D_dev, const double* v_dev, double* result);
/* Verdict of the last reduce_qr on this plan (synchronises): BLS_OK / BLS_NOT_PD (failed_block 1-based) / BLS_EINVAL. */
int bls_qr_query_status(bls_qr_plan* plan, int64_t* failed_block);
/* Device kernel launches issued on this plan since the previous call (no counterpart in the reference). */
int64_t bls_qr_plan_counters(bls_qr_plan* plan);
/* qr_backsubstitute! (src/qr_reduced.jl:24-93): x_e = U^-1 (q - B x_r) per eliminated block, in double. */
int bls_qr_backsubstitute(bls_qr_plan* plan, int dtype, double* x_e_dev, const double* x_r_dev, const void* F_dev,
                          const double* Fr_dev);
/* reduced_normal_sparse! / reduced_normal_dense! (src/qr_reduced.jl:409-480): S = J~'J~ (upper blocks; the sparse form
 * on the plan's pattern, the dense form column-major nr x nr) and g_S = J~'r~ from the factored tables. */
int bls_reduced_normal_sparse(bls_qr_plan* plan, int dtype, void* S_nzval_dev, double* g_S_dev, const void* F_dev,
                              const double* Fr_dev);
int bls_reduced_normal_dense(bls_qr_plan* plan, int dtype, void* S_dev, double* g_S_dev, const void* F_dev,
                             const double* Fr_dev);
/* reduced_diagonal_blocks! (src/qr_reduced.jl:484-512): the full d_r x d_r diagonal blocks of J~'J~ at doffsets. */
int bls_reduced_diagonal_blocks(bls_qr_plan* plan, int dtype, void* D_dev, const void* F_dev);
/* The reduced problem written out (src/qr_reduced.jl:227-370), from the factored tables F / Fr. reduced_residual!:
 * rt = r~ (reduced_nrows FP64 entries, tables in order, each its bottom residual rows). reduced_jacobian! dense: Jt =
 * J~, column-major nrows x ncols = reduced_nrows x nr, zero outside the tables' runs, and rt = r~. Sparse: nzval (on
 * the device) of the CSC pattern of build_reduced_jacobian_pattern, which the caller passes (colptr[ncols + 1] and
 * rowval, 0-based, on the host) and which is checked before any work as the reference checks it: a wrong size or rt
 * length is BLS_EDIM (DimensionMismatch), a column of the wrong height or a run that starts at the wrong row BLS_EINVAL
 * (ArgumentError, messages 1-based). */
/* reduced_mul! (src/qr_reduced.jl:159-192): y = J~ v (ny = reduced_nrows, nv = nr); reduced_tmul!
 * (src/qr_reduced.jl:194-223): g = J~' w (ng = nr, nw = reduced_nrows); FP64 vectors, products accumulated in FP64,
 * applied from the factored tables without forming J~ (the per-iteration work of an LSMR solve of the reduced
 * problem). A wrong length is BLS_EDIM. reduced_tmul! keeps a scratch of n_entries x (largest retained block) doubles
 * in the plan, allocated at its first call; its sums are deterministic (no atomics). */
int bls_reduced_mul(bls_qr_plan* plan, int dtype, const void* F_dev, const double* v_dev, int64_t nv, double* y_dev, int64_t ny);
int bls_reduced_tmul(bls_qr_plan* plan, int dtype, const void* F_dev, const double* w_dev, int64_t nw, double* g_dev, int64_t ng);
int bls_reduced_residual(bls_qr_plan* plan, const double* Fr_dev, double* rt_dev, int64_t n_rt);
int bls_reduced_jacobian_dense(bls_qr_plan* plan, int dtype, const void* F_dev, const double* Fr_dev, void* Jt_dev, int64_t nrows,
                               int64_t ncols, double* rt_dev, int64_t n_rt);
int bls_reduced_jacobian_sparse(bls_qr_plan* plan, int dtype, const void* F_dev, const double* Fr_dev, int64_t nrows, int64_t ncols,
                                const int64_t* colptr, const int64_t* rowval, void* nzval_dev, double* rt_dev, int64_t n_rt);

/* LSMR on the reduced problem (replaces KrylovExt's solve!, ext/KrylovExt.jl:97-132, with reduced_mul! / reduced_tmul! /
 * reduced_diagonal_blocks! of src/qr_reduced.jl as its operator): x_dev (nr doubles) = argmin || A x - [r~; 0] ||,
 * A = [J~; diag(sqrt(lambda s_r))], J~ and r~ read from the factored tables F_dev / Fr_dev of the last reduce_qr, block-
 * Jacobi preconditioned by the diagonal blocks of A'A (Krylov's N = D^-1). s_r_dev NULL: all ones. Stopping by the
 * tolerances atol, btol and conlim of Fong & Saunders' LSMR (the reference passes sqrt(eps(T)) for the three and
 * 1/sqrt(eps(T)) for conlim); itmax < 0: reduced_nrows + nr. The vectors and the block factors are FP64 for both dtypes.
 * Returns BLS_OK (solved: istop 1, 2, 4 or 5), BLS_NOT_PD where the reference's solve! returns NotPositiveDefinite (a
 * non-finite r~, lambda == 0 with fewer reduced rows than nr, a diagonal block that is not positive definite, cond(A)
 * above conlim: istop 3 or 6, a non-finite x), BLS_NOT_CONVERGED at itmax (istop 7; also NotPositiveDefinite there).
 * iterations, istop, stats (5 doubles: the estimates of ||r||, ||A'r||, ||A||, cond(A) of the preconditioned operator,
 * and ||x||) may be NULL. The plan keeps the solve's vectors and scratch (allocated at its first call); the call
 * synchronises the context's stream twice per iteration to read the norms. */
int bls_lsmr_reduced(bls_qr_plan* plan, int dtype, const void* F_dev, const double* Fr_dev, double lambda, const double* s_r_dev,
                     double* x_dev, int64_t nx, double atol, double btol, double conlim, int64_t itmax, int64_t* iterations,
                     int* istop, double* stats);

/* ---------------------------------------------------------------------------------------------------------------
 * Block-Jacobi (src/diagonal_blocks.jl:6-61) on a flat array of square diagonal blocks (block b, d_b x d_b column-major,
 * after the blocks before it), as reduced_diagonal_blocks! writes them. d_b <= 16.
 * ------------------------------------------------------------------------------------------------------------- */
int bls_block_jacobi_create(bls_ctx* ctx, int64_t nblocks, const int64_t* dims, bls_block_jacobi** out);
int bls_block_jacobi_destroy(bls_block_jacobi* bj);
/* factor_diagonal_blocks!(D, dims) -> Bool: each block's Cholesky factor L in place in its lower triangle. BLS_OK, or
 * BLS_NOT_PD with failed_block = the lowest block (1-based) that is not positive definite or not finite. Synchronises. */
int bls_factor_diagonal_blocks(bls_block_jacobi* bj, int dtype, void* D_dev, int64_t* failed_block);
/* solve_diagonal_blocks!(y, D, dims, x): y = (L L')^-1 x block by block (y may be x); x, y double. */
int bls_solve_diagonal_blocks(bls_block_jacobi* bj, int dtype, double* y_dev, const void* D_dev, const double* x_dev);

/* ---------------------------------------------------------------------------------------------------------------
 * PCG on the reduced system S x = g (no counterpart in the reference, which solves it with CHOLMOD / LDLFactorizations,
 * src/schur_linear_systems.jl:362-406; its iterative path is LSMR on J~ with the same block-Jacobi preconditioner,
 * ext/KrylovExt.jl:97-132). S: the upper block triangle on build_schur_pattern's pattern, as reduce_schur_sparse!
 * leaves it. x, g double.
 * ------------------------------------------------------------------------------------------------------------- */
int bls_pcg_plan_create(bls_ctx* ctx, int64_t nrblocks, const int64_t* r_dims, const int64_t* block_colptr,
                        const int64_t* block_rowval, const int64_t* block_row_offsets, const int64_t* col_heights,
                        const int64_t* S_colptr, bls_pcg_plan** out);
int bls_pcg_plan_destroy(bls_pcg_plan* plan);
/* y = S x with S symmetric (its upper blocks mirrored), FP64 products. */
int bls_spmv_sym(bls_pcg_plan* plan, int dtype, const void* S_nzval_dev, const double* x_dev, double* y_dev);
/* The full d_r x d_r diagonal blocks of S (upper triangles mirrored) as doubles, block after block. */
int bls_extract_diagonal_blocks(bls_pcg_plan* plan, int dtype, const void* S_nzval_dev, double* D_dev);
/* PCG from the initial x to ||g - S x||_2 <= tol ||g||_2, checked on an explicit FP64 residual (restarted from x while
 * the recursive residual has drifted: iterative refinement), preconditioned by the block-Jacobi factorisation of S's
 * diagonal blocks. use_graph: replay runs of iterations as one CUDA graph. Returns BLS_OK, BLS_NOT_CONVERGED (maxit
 * reached; x is the last iterate) or BLS_NOT_PD (failed_block = the lowest diagonal block of S, 1-based, that is not
 * positive definite). iterations and rel_residual report the run. */
int bls_pcg_solve(bls_pcg_plan* plan, int dtype, const void* S_nzval_dev, const double* g_dev, double* x_dev, double tol,
                  int64_t maxit, int use_graph, int64_t* iterations, double* rel_residual, int64_t* failed_block);
/* Mixed-precision reduced solve with iterative refinement against the FP64 reduced operator (no counterpart in the
 * reference): x solves A x = g, A = S0 + lambda diag(scaling_r) - C' E^-1 C applied in FP64 (S0 = R on S's pattern,
 * e.g. bls_reset_schur_sparse with lambda = 0; C and E^-1 as in bls_schur_apply_elimination, from `schur`'s last
 * reduction), while every inner PCG iteration reads only the stored reduced S (e.g. the FP32 reduction of the same
 * system): x = 0, r = g; repeat d = PCG(S, r) to inner_tol, x += d, r = g - A x, until ||r|| <= tol ||g|| or
 * max_outer corrections. Both plans must be on the same context. Returns BLS_OK, BLS_NOT_CONVERGED or BLS_NOT_PD
 * (a diagonal block of S); outer_iterations / inner_iterations count the corrections and the PCG iterations,
 * rel_residual is the last ||g - A x|| / ||g||. */
int bls_pcg_solve_refined(bls_pcg_plan* plan, bls_schur_plan* schur, int dtype, const void* S_nzval_dev, const void* S0_nzval_dev,
                          const double* scaling_r_dev, double lambda, const void* C_data_dev, const double* g_dev, double* x_dev,
                          double tol, double inner_tol, int64_t max_outer, int64_t inner_maxit, int64_t* outer_iterations,
                          int64_t* inner_iterations, double* rel_residual, int64_t* failed_block);
/* Dense reduced solve (the reference hands a dense S to DampedLinearSolve's Cholesky, src/schur_linear_systems.jl:
 * 312-320): a solver for n x n systems (n <= 16384) owning an FP64 working matrix. bls_dense_cholesky reads S
 * (dtype, column-major, its upper triangle: reduce_schur_dense!'s output) and factors it as L L' in FP64; a pivot that
 * is not positive returns BLS_NOT_PD with failed_column = its column, 1-based. bls_dense_cholesky_solve: x = S^-1 g
 * (FP64 device vectors) from the last successful factorisation. */
typedef struct bls_dense_solver bls_dense_solver;
int bls_dense_solver_create(bls_ctx* ctx, int64_t n, bls_dense_solver** out);
int bls_dense_solver_destroy(bls_dense_solver* solver);
int bls_dense_cholesky(bls_dense_solver* solver, int dtype, const void* S_dev, int64_t* failed_column);
int bls_dense_cholesky_solve(bls_dense_solver* solver, const double* g_dev, double* x_dev);

/* The same factorisation of S + lambda diag(s_r) (s_r a device vector of n FP64 entries, added to the diagonal in FP64
 * as S is read): the damped reduced normal equations of the QR route, J~'J~ from bls_reduced_normal_dense plus
 * lambda s_r (src/qr_linear_systems.jl:315-322). lambda must be finite and non-negative (BLS_EINVAL). */
int bls_dense_cholesky_shifted(bls_dense_solver* solver, int dtype, const void* S_dev, double lambda, const double* s_r_dev,
                               int64_t* failed_column);

/* prepare_scale! (src/conditioning.jl:60-87) of an EliminationConditioning: s[n] = the conditioning scale of each
 * variable (conditioning_scale, :29-36: the power of two nearest on a log scale to 1/(1e-12 + sqrt|d_j + lambda sc_j|),
 * at least floatmin of dtype, 1 for a non-finite entry), computed for every variable when stale is set, else only when
 * some variable's |d_j + lambda sc_j| s_j^2 lies outside [2^-16, 2^16] and its scale would change; lambda below 0 counts
 * as 0. d, sc, s device vectors. *recomputed (may be NULL; synchronises) = whether s was rewritten. Bit-identical to
 * the reference's scales. */
int bls_prepare_scale(bls_ctx* ctx, int dtype, int64_t n, const double* d_dev, double lambda, const double* sc_dev, double* s_dev,
                      int stale, int* recomputed);

/* Device kernel launches issued on this plan since the previous call (no counterpart in the reference). */
int64_t bls_pcg_plan_counters(bls_pcg_plan* plan);
/* Replace the block-Jacobi solve in later bls_pcg_solve calls by z_b = B_b r_b with the dense symmetric positive definite
 * blocks B (double, d_r x d_r column-major per retained block, block after block, in device memory the caller keeps);
 * NULL restores block-Jacobi. */
int bls_pcg_set_preconditioner(bls_pcg_plan* plan, const double* blocks_dev);

/* ---------------------------------------------------------------------------------------------------------------
 * Learned block preconditioner (no counterpart in the reference): a 3-layer, width-64 graph network over the camera
 * covisibility graph of S that predicts a lower-triangular correction T_b per 6 x 6 block; the preconditioner block is
 * L_b^-T (I + T_b)' (I + T_b) L_b^-1 with L_b the Cholesky factor of S_bb (T = 0 is block-Jacobi). Parameters: a float
 * vector of bls_gnn_param_count() entries (layout in csrc/gnn.cu). Retained blocks must all be 6 x 6.
 * ------------------------------------------------------------------------------------------------------------- */
int64_t bls_gnn_param_count(void);
int bls_gnn_create(bls_pcg_plan* plan, const int64_t* block_colptr, const int64_t* block_rowval, const int64_t* block_row_offsets,
                   const int64_t* col_heights, const int64_t* S_colptr, bls_gnn** out);
int bls_gnn_destroy(bls_gnn* g);
/* Graph features of S (its block-Jacobi factors, normalised couplings, node features). BLS_NOT_PD: a diagonal block of S
 * is not positive definite (failed_block, 1-based). */
int bls_gnn_prepare(bls_gnn* g, int dtype, const void* S_nzval_dev, int64_t* failed_block);
/* Inference (bf16 != 0: BF16 activations and weights, FP32 accumulation; else FP32): the preconditioner blocks
 * (36 doubles per retained block) into blocks_dev. */
int bls_gnn_forward(bls_gnn* g, const float* params_dev, int bf16, double* blocks_dev);
/* Copies of the last forward's outputs t (21 floats per block), the node features (8 floats per block) and the edge
 * weights (one double per stored off-diagonal block); any may be NULL. */
int bls_gnn_outputs(bls_gnn* g, float* t_dev, float* features_dev, double* edge_norms_dev);
int64_t bls_gnn_edge_count(bls_gnn* g);
/* Training loss mean_p ||G S^ G' z_p - z_p||^2 / ||z_p||^2 (S^ = L^-1 S L^-T) over nprobes probe vectors (double,
 * nr each, one after another) and its gradient (float, bls_gnn_param_count() entries, overwritten). FP32 network. */
int bls_gnn_loss_grad(bls_gnn* g, int dtype, const void* S_nzval_dev, const float* params_dev, const double* probes_dev,
                      int64_t nprobes, double* loss, float* grad_dev);
/* One Adam step on n parameters (step counts from 1). */
int bls_adam_step(bls_ctx* ctx, float* params_dev, const float* grad_dev, float* m_dev, float* v_dev, int64_t n, float lr,
                  float beta1, float beta2, float eps, int64_t step);

/* copyto!(csc, bsm, scatter_map) (src/SparseBlockLinearSystem.jl:356-362): dest[i] = src[map[i]], i < n. */
int bls_scatter_copy(bls_ctx* ctx, int dtype, void* dest_dev, const void* src_dev, const int64_t* map_dev, int64_t n);

/* symmetrifyfull!(mat, bsm, blocks) (src/SparseBlockLinearSystem.jl:299-341): the dense symmetric matrix of a
 * block-square SparseBlockLinearSystem, each block (r, c) copied to its place and, for r != c, transposed to (c, r).
 * The system is given on the host by its nb block sizes and its indicestransposed as a CSC over block rows: for k in
 * [it_colptr[r], it_colptr[r + 1]), block (r, it_rowval[k]) starts at data[it_nzval[k]] (column-major, blocksizes[r]
 * x blocksizes[c]); for the retained part R of a Schur pattern these are r_dims, block_colptr, block_rowval and
 * R_block_start. data and mat (m x m, column-major, zero outside the blocks) are device buffers of dtype. blocks:
 * the 0-based blocks to include, in the order they take in mat (NULL: all, in order; nblocks is then ignored).
 * Errors, before any write: a block out of range (the reference's BoundsError) or listed twice BLS_EINVAL; m other
 * than the total size of the included blocks (DimensionMismatch) BLS_EDIM. Where blocks (r, c) and (c, r) are both
 * present, the one later in indicestransposed is the one written, as the reference's loop leaves it. */
int bls_symmetrify_full(bls_ctx* ctx, int dtype, int64_t nb, const int64_t* blocksizes, const int64_t* it_colptr,
                        const int64_t* it_rowval, const int64_t* it_nzval, const void* data_dev, const int64_t* blocks,
                        int64_t nblocks, void* mat_dev, int64_t m);

#ifdef __cplusplus
}
#endif
#endif /* BLSGPU_H */
