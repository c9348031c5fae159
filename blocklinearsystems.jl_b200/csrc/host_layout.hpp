// Host-side layout types shared by the C ABI and the layout builders (0-based throughout).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/blsgpu.h"

namespace bls {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// SchurStructure (src/schur_structure.jl:50-68) plus the workspace index of SchurReductionWorkspace
// (src/schur_reduction.jl:22-25).
struct Structure {
  int64_t nr = 0, ne = 0, nrblocks = 0, neblocks = 0, nchunks = 1, min_work = 4096, max_coupled_dim = 0;
  int64_t E_length = 0, C_length = 0;
  std::vector<int64_t> r_dims, e_dims, boffsets_r, boffsets_e, eoffsets, eliminated_ptr, entry_retained, coffsets, order;
  std::vector<std::pair<int64_t, int64_t>> retained_pairs;
  std::vector<int64_t> e_run_first;   // first block of each run of equal e_dims, then neblocks
  std::vector<int64_t> chunks;        // per run, nchunks half-open ranges (first, stop)
  std::vector<int64_t> retained_ptr, retained_entry, entry_eliminated;
  std::vector<int64_t> col_chunks;    // nchunks half-open ranges of retained blocks
};

// build_schur_pattern's result (src/schur_structure.jl:314-322) and the retained storage laid out on it.
struct Pattern {
  std::vector<int64_t> block_colptr, block_rowval, block_row_offsets, col_heights, S_colptr, S_rowval, diag_inds;
  std::vector<int64_t> R_block_start;
  int64_t R_length = 0;
};

std::vector<int64_t> partition_columns(const std::vector<int64_t>& retained_ptr, int64_t K);
void finish_structure(Structure& st, const std::vector<std::vector<int64_t>>& couplings);
Structure structure_positional(const std::vector<int64_t>& r_dims, const std::vector<int64_t>& e_dims,
                               const std::vector<std::vector<int64_t>>& couplings, int64_t nchunks, int64_t min_work);
Structure structure_from_description(int64_t n, const int64_t* blocksizes, int64_t K, const int64_t* rb_ptr,
                                     const int64_t* rb_idx, const uint8_t* eliminated, int64_t nchunks, int64_t min_work,
                                     const int64_t* rowblocksizes = nullptr);
Pattern build_pattern(const Structure& st, const std::vector<std::pair<int64_t, int64_t>>& extra);
std::vector<int64_t> build_r_to_s(const Structure& st, const Pattern& P);
int64_t sparse_indices(const Structure& st, const Pattern& P, bool symmetric, int64_t* colptr, int64_t* rowval, int64_t* map);

}  // namespace bls

namespace bls {

// SchurJacobianStructure (src/schur_jacobian.jl:30-57): one table per eliminated block (its rows, then d_e damping rows;
// columns: the coupled retained blocks' columns, then the d_e eliminated columns; the residual is a separate FP64 column),
// then one table per free group of row blocks that touch no eliminated block.
struct QRStructure {
  Structure schur;
  int64_t ntables = 0;
  std::vector<int64_t> e_rows, free_rows, table_nrows, table_ncols, table_top, table_offsets, raw_offsets, residual_offsets;
  std::vector<int64_t> table_ptr, entry_retained, entry_col, entry_table, retained_ptr, retained_entry, reduced_offsets, doffsets;
  std::vector<int64_t> col_chunks, row_table, row_first, row_nrows, row_ptr, row_blocks;
};

QRStructure qr_structure(const Structure& st, const std::vector<int64_t>& e_rows, const std::vector<int64_t>& free_rows,
                         const std::vector<std::vector<int64_t>>& free_retained, int64_t nchunks);
QRStructure qr_structure_from_description(int64_t n, const int64_t* blocksizes, int64_t K, const int64_t* rb_ptr, const int64_t* rb_idx,
                                          const int64_t* rowblocksizes, const uint8_t* eliminated, int64_t nchunks, int64_t min_work);

}  // namespace bls
