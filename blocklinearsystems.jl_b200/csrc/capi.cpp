// C ABI of libblsgpu: contexts, errors and the host-side layout (structure, pattern, maps).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>

#include "common.cuh"

namespace bls {
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
}  // namespace bls

struct bls_structure : bls::Structure {};
struct bls_pattern : bls::Pattern {};
struct bls_qr_structure : bls::QRStructure {};

using namespace bls;

#define BLS_GUARD(...)                         \
  try {                                        \
    __VA_ARGS__                                \
  } catch (const bls::Error& e) {              \
    bls::set_error(e.what());                  \
    return e.code;                             \
  } catch (const std::bad_alloc&) {            \
    bls::set_error("out of host memory");      \
    return BLS_ENOMEM;                         \
  } catch (const std::exception& e) {          \
    bls::set_error(e.what());                  \
    return BLS_EINVAL;                         \
  }

static int64_t put(int64_t* out, const std::vector<int64_t>& v) {
  if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(int64_t));
  return (int64_t)v.size();
}

extern "C" {

int bls_version(void) { return 1; }
const char* bls_last_error(void) { return bls::g_last_error.c_str(); }

int bls_ctx_create(int device, bls_ctx** out) {
  BLS_GUARD({
    if (!out) throw Error(BLS_EINVAL, "null argument");
    int n = 0;
    BLS_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw Error(BLS_EINVAL, "no CUDA device " + std::to_string(device));
    BLS_CUDA(cudaSetDevice(device));
    auto* c = new bls_ctx();
    c->device = device;
    c->stream = nullptr;
    *out = c;
    return BLS_OK;
  })
}

int bls_ctx_destroy(bls_ctx* ctx) {
  if (ctx && ctx->flag) cudaFree(ctx->flag);
  delete ctx;
  return BLS_OK;
}

int bls_ctx_set_stream(bls_ctx* ctx, void* stream) {
  if (!ctx) return BLS_EINVAL;
  ctx->stream = static_cast<cudaStream_t>(stream);
  return BLS_OK;
}

int bls_ctx_synchronize(bls_ctx* ctx) {
  BLS_GUARD({
    BLS_CUDA(cudaStreamSynchronize(ctx->stream));
    return BLS_OK;
  })
}

int bls_structure_from_description(int64_t nblocks, const int64_t* blocksizes, int64_t nrowblocks, const int64_t* rowblock_ptr,
                                   const int64_t* rowblock_idx, const uint8_t* eliminated, int64_t nchunks, int64_t min_work,
                                   bls_structure** out) {
  BLS_GUARD({
    if (!out || (nblocks > 0 && (!blocksizes || !eliminated)) || (nrowblocks > 0 && (!rowblock_ptr || !rowblock_idx)))
      throw Error(BLS_EINVAL, "null argument");
    auto* s = new bls_structure();
    try {
      static_cast<Structure&>(*s) = structure_from_description(nblocks, blocksizes, nrowblocks, rowblock_ptr, rowblock_idx, eliminated, nchunks, min_work);
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
    return BLS_OK;
  })
}

int bls_structure_positional(int64_t nrblocks, const int64_t* r_dims, int64_t neblocks, const int64_t* e_dims, const int64_t* coupling_ptr,
                             const int64_t* coupling_idx, int64_t nchunks, int64_t min_work, bls_structure** out) {
  BLS_GUARD({
    std::vector<std::vector<int64_t>> coup(neblocks);
    for (int64_t e = 0; e < neblocks; ++e) coup[e].assign(coupling_idx + coupling_ptr[e], coupling_idx + coupling_ptr[e + 1]);
    auto* s = new bls_structure();
    try {
      static_cast<Structure&>(*s) = structure_positional(std::vector<int64_t>(r_dims, r_dims + nrblocks), std::vector<int64_t>(e_dims, e_dims + neblocks), coup, nchunks, min_work);
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
    return BLS_OK;
  })
}

int64_t bls_structure_field(const bls_structure* st, const char* name, int64_t* out) {
  if (!st || !name) return -1;
  const std::string f(name);
  auto scalar = [&](int64_t v) { if (out) out[0] = v; return (int64_t)1; };
  if (f == "nr") return scalar(st->nr);
  if (f == "ne") return scalar(st->ne);
  if (f == "nrblocks") return scalar(st->nrblocks);
  if (f == "neblocks") return scalar(st->neblocks);
  if (f == "max_coupled_dim") return scalar(st->max_coupled_dim);
  if (f == "E_length") return scalar(st->E_length);
  if (f == "C_length") return scalar(st->C_length);
  if (f == "nchunks") return scalar(st->nchunks);
  if (f == "min_work") return scalar(st->min_work);
  if (f == "r_dims") return put(out, st->r_dims);
  if (f == "e_dims") return put(out, st->e_dims);
  if (f == "boffsets_r") return put(out, st->boffsets_r);
  if (f == "boffsets_e") return put(out, st->boffsets_e);
  if (f == "eoffsets") return put(out, st->eoffsets);
  if (f == "eliminated_ptr") return put(out, st->eliminated_ptr);
  if (f == "entry_retained") return put(out, st->entry_retained);
  if (f == "coffsets") return put(out, st->coffsets);
  if (f == "order") return put(out, st->order);
  if (f == "chunks") return put(out, st->chunks);
  if (f == "retained_ptr") return put(out, st->retained_ptr);
  if (f == "retained_entry") return put(out, st->retained_entry);
  if (f == "entry_eliminated") return put(out, st->entry_eliminated);
  if (f == "col_chunks") return put(out, st->col_chunks);
  if (f == "retained_pairs") {
    std::vector<int64_t> v;
    for (auto& p : st->retained_pairs) { v.push_back(p.first); v.push_back(p.second); }
    return put(out, v);
  }
  return -1;
}

int bls_structure_destroy(bls_structure* st) {
  delete st;
  return BLS_OK;
}

int bls_schur_pattern_build(const bls_structure* st, int64_t nextra, const int64_t* extra_pairs, bls_pattern** out) {
  BLS_GUARD({
    if (!st || !out) throw Error(BLS_EINVAL, "null argument");
    std::vector<std::pair<int64_t, int64_t>> ex;
    for (int64_t i = 0; i < nextra; ++i) ex.push_back({extra_pairs[2 * i], extra_pairs[2 * i + 1]});
    auto* p = new bls_pattern();
    try {
      static_cast<Pattern&>(*p) = build_pattern(*st, ex);
    } catch (...) {
      delete p;
      throw;
    }
    *out = p;
    return BLS_OK;
  })
}

int64_t bls_pattern_field(const bls_pattern* p, const char* name, int64_t* out) {
  if (!p || !name) return -1;
  const std::string f(name);
  if (f == "block_colptr") return put(out, p->block_colptr);
  if (f == "block_rowval") return put(out, p->block_rowval);
  if (f == "block_row_offsets") return put(out, p->block_row_offsets);
  if (f == "col_heights") return put(out, p->col_heights);
  if (f == "S_colptr") return put(out, p->S_colptr);
  if (f == "S_rowval") return put(out, p->S_rowval);
  if (f == "diag_inds") return put(out, p->diag_inds);
  if (f == "R_block_start") return put(out, p->R_block_start);
  if (f == "R_length") { if (out) out[0] = p->R_length; return 1; }
  return -1;
}

int bls_pattern_destroy(bls_pattern* p) {
  delete p;
  return BLS_OK;
}

int bls_build_r_to_s_map(const bls_structure* st, const bls_pattern* p, int64_t* out) {
  BLS_GUARD({
    if (!st || !p || !out) throw Error(BLS_EINVAL, "null argument");
    std::vector<int64_t> m = build_r_to_s(*st, *p);
    put(out, m);
    return BLS_OK;
  })
}

// find_in_column (src/schur_structure.jl:355-361): the position of `row` in column j of S (rows sorted), or -1
static int64_t find_in_column(const int64_t* S_colptr, const int64_t* S_rowval, int64_t row, int64_t j) {
  const int64_t* lo = S_rowval + S_colptr[j];
  const int64_t* hi = S_rowval + S_colptr[j + 1];
  const int64_t* f = std::lower_bound(lo, hi, row);
  return (f != hi && *f == row) ? (int64_t)(f - S_rowval) : -1;
}

int bls_r_to_s_map_csc(int64_t ncols, const int64_t* R_colptr, const int64_t* R_rowval, const int64_t* S_colptr, const int64_t* S_rowval,
                       int64_t* out) {
  BLS_GUARD({
    if (ncols < 0 || (ncols > 0 && (!R_colptr || !S_colptr)) || (ncols > 0 && R_colptr[ncols] > 0 && (!R_rowval || !out)))
      throw Error(BLS_EINVAL, "null argument");
    const int64_t nnz = ncols > 0 ? R_colptr[ncols] : 0;
    std::vector<int64_t> m((size_t)nnz);
    for (int64_t j = 0; j < ncols; ++j)
      for (int64_t k = R_colptr[j]; k < R_colptr[j + 1]; ++k) {
        const int64_t i = R_rowval[k], s_k = find_in_column(S_colptr, S_rowval, i, j);
        if (s_k < 0)
          throw Error(BLS_EINVAL, "R entry (" + std::to_string(i + 1) + ", " + std::to_string(j + 1) + ") is not present in the sparsity pattern of S");
        m[k] = s_k;
      }
    if (nnz > 0) std::memcpy(out, m.data(), sizeof(int64_t) * (size_t)nnz);
    return BLS_OK;
  })
}

int bls_r_to_s_map_blocks_csc(int64_t nb, const int64_t* blocksizes, const int64_t* it_colptr, const int64_t* it_rowval, const int64_t* it_nzval,
                              int64_t data_len, const int64_t* S_colptr, const int64_t* S_rowval, const int64_t* boffsets_r, int64_t* out) {
  BLS_GUARD({
    if (nb < 0 || data_len < 0 || (nb > 0 && (!blocksizes || !it_colptr || !S_colptr || !boffsets_r)) || (data_len > 0 && !out))
      throw Error(BLS_EINVAL, "null argument");
    std::vector<int64_t> m((size_t)data_len, -1);
    // findnz(indicestransposed): block rows brow in order, then their block columns
    for (int64_t brow = 0; brow < nb; ++brow)
      for (int64_t k = it_colptr[brow]; k < it_colptr[brow + 1]; ++k) {
        const int64_t bcol = it_rowval[k], start = it_nzval[k], drow = blocksizes[brow], dcol = blocksizes[bcol];
        if (bcol < 0 || bcol >= nb || start < 0 || start + drow * dcol > data_len) throw Error(BLS_EINVAL, "indicestransposed is malformed");
        if (brow == bcol) {
          for (int64_t col = 0; col < dcol; ++col) {
            const int64_t scol = boffsets_r[brow] + col;
            for (int64_t row = 0; row <= col; ++row) {
              const int64_t srow = boffsets_r[brow] + row, s_k = find_in_column(S_colptr, S_rowval, srow, scol);
              if (s_k < 0)
                throw Error(BLS_EINVAL, "Entry (" + std::to_string(srow + 1) + ", " + std::to_string(scol + 1) +
                                            ") of a diagonal block of R is not present in the sparsity pattern of S");
              m[start + col * drow + row] = s_k;
            }
          }
        } else if (brow > bcol) {
          for (int64_t col = 0; col < dcol; ++col) {
            const int64_t srow = boffsets_r[bcol] + col;
            for (int64_t row = 0; row < drow; ++row) {
              const int64_t scol = boffsets_r[brow] + row, s_k = find_in_column(S_colptr, S_rowval, srow, scol);
              if (s_k < 0)
                throw Error(BLS_EINVAL, "Entry (" + std::to_string(srow + 1) + ", " + std::to_string(scol + 1) +
                                            ") of R is not present in the sparsity pattern of S");
              m[start + col * drow + row] = s_k;
            }
          }
        }
      }
    if (data_len > 0) std::memcpy(out, m.data(), sizeof(int64_t) * (size_t)data_len);
    return BLS_OK;
  })
}

int64_t bls_sparse_indices(const bls_structure* st, const bls_pattern* p, int symmetric, int64_t* colptr, int64_t* rowval, int64_t* map) {
  BLS_GUARD({
    if (!st || !p) throw Error(BLS_EINVAL, "null argument");
    return sparse_indices(*st, *p, symmetric != 0, colptr, rowval, map);
  })
}

int bls_qr_structure_from_description(int64_t nblocks, const int64_t* blocksizes, int64_t nrowblocks, const int64_t* rowblock_ptr,
                                      const int64_t* rowblock_idx, const int64_t* rowblocksizes, const uint8_t* eliminated, int64_t nchunks,
                                      int64_t min_work, bls_qr_structure** out) {
  BLS_GUARD({
    if (!out || (nblocks > 0 && (!blocksizes || !eliminated)) || (nrowblocks > 0 && (!rowblock_ptr || !rowblock_idx || !rowblocksizes)))
      throw Error(BLS_EINVAL, "null argument");
    auto* q = new bls_qr_structure();
    try {
      static_cast<QRStructure&>(*q) = qr_structure_from_description(nblocks, blocksizes, nrowblocks, rowblock_ptr, rowblock_idx, rowblocksizes,
                                                                    eliminated, nchunks, min_work);
    } catch (...) {
      delete q;
      throw;
    }
    *out = q;
    return BLS_OK;
  })
}

int bls_qr_structure_positional(const bls_structure* st, const int64_t* e_rows, int64_t nfree, const int64_t* free_rows, const int64_t* free_ptr,
                                const int64_t* free_idx, int64_t nchunks, bls_qr_structure** out) {
  BLS_GUARD({
    if (!st || !out || (st->neblocks > 0 && !e_rows) || (nfree > 0 && (!free_rows || !free_ptr || !free_idx))) throw Error(BLS_EINVAL, "null argument");
    std::vector<std::vector<int64_t>> fr(nfree);
    for (int64_t g = 0; g < nfree; ++g) fr[g].assign(free_idx + free_ptr[g], free_idx + free_ptr[g + 1]);
    auto* q = new bls_qr_structure();
    try {
      static_cast<QRStructure&>(*q) = qr_structure(*st, std::vector<int64_t>(e_rows, e_rows + st->neblocks),
                                                   std::vector<int64_t>(free_rows, free_rows + nfree), fr, nchunks);
    } catch (...) {
      delete q;
      throw;
    }
    *out = q;
    return BLS_OK;
  })
}

int64_t bls_reduced_jacobian_pattern(const bls_qr_structure* q, int64_t* colptr, int64_t* rowval) {
  if (!q) {
    bls::set_error("structure is NULL");
    return BLS_EINVAL;
  }
  const Structure& st = q->schur;
  std::vector<int64_t> cp((size_t)st.nr + 1, 0);
  auto height = [&](int64_t r) {
    int64_t h = 0;
    for (int64_t k = q->retained_ptr[r]; k < q->retained_ptr[r + 1]; ++k) {
      const int64_t t = q->entry_table[q->retained_entry[k]];
      h += q->table_nrows[t] - q->table_top[t];
    }
    return h;
  };
  for (int64_t r = 0; r < st.nrblocks; ++r) {
    const int64_t h = height(r), ro = st.boffsets_r[r];
    for (int64_t j = 0; j < st.r_dims[r]; ++j) cp[ro + j + 1] = cp[ro + j] + h;
  }
  const int64_t nnz = cp[st.nr];
  if (colptr) std::memcpy(colptr, cp.data(), sizeof(int64_t) * cp.size());
  if (rowval)
    for (int64_t r = 0; r < st.nrblocks; ++r)
      for (int64_t j = 0; j < st.r_dims[r]; ++j) {
        int64_t p = cp[st.boffsets_r[r] + j];
        for (int64_t k = q->retained_ptr[r]; k < q->retained_ptr[r + 1]; ++k) {
          const int64_t t = q->entry_table[q->retained_entry[k]];
          for (int64_t i = 0; i < q->table_nrows[t] - q->table_top[t]; ++i) rowval[p++] = q->reduced_offsets[t] + i;
        }
      }
  return nnz;
}

int64_t bls_qr_structure_field(const bls_qr_structure* q, const char* name, int64_t* out) {
  if (!q || !name) return -1;
  const std::string f(name);
  auto scalar = [&](int64_t v) { if (out) out[0] = v; return (int64_t)1; };
  if (f == "ntables") return scalar(q->ntables);
  if (f == "raw_length") return scalar(q->raw_offsets.back());
  if (f == "residual_length") return scalar(q->residual_offsets.back());
  if (f == "e_rows") return put(out, q->e_rows);
  if (f == "free_rows") return put(out, q->free_rows);
  if (f == "table_nrows") return put(out, q->table_nrows);
  if (f == "table_ncols") return put(out, q->table_ncols);
  if (f == "table_top") return put(out, q->table_top);
  if (f == "table_offsets") return put(out, q->table_offsets);
  if (f == "raw_offsets") return put(out, q->raw_offsets);
  if (f == "residual_offsets") return put(out, q->residual_offsets);
  if (f == "reduced_offsets") return put(out, q->reduced_offsets);
  if (f == "table_ptr") return put(out, q->table_ptr);
  if (f == "entry_retained") return put(out, q->entry_retained);
  if (f == "entry_col") return put(out, q->entry_col);
  if (f == "entry_table") return put(out, q->entry_table);
  if (f == "retained_ptr") return put(out, q->retained_ptr);
  if (f == "retained_entry") return put(out, q->retained_entry);
  if (f == "doffsets") return put(out, q->doffsets);
  if (f == "col_chunks") return put(out, q->col_chunks);
  if (f == "row_table") return put(out, q->row_table);
  if (f == "row_first") return put(out, q->row_first);
  if (f == "row_nrows") return put(out, q->row_nrows);
  if (f == "row_ptr") return put(out, q->row_ptr);
  if (f == "row_blocks") return put(out, q->row_blocks);
  return -1;
}

int bls_qr_structure_schur(const bls_qr_structure* q, bls_structure** out) {
  BLS_GUARD({
    if (!q || !out) throw Error(BLS_EINVAL, "null argument");
    auto* s = new bls_structure();
    static_cast<Structure&>(*s) = q->schur;
    *out = s;
    return BLS_OK;
  })
}

int bls_qr_structure_destroy(bls_qr_structure* q) {
  delete q;
  return BLS_OK;
}


int bls_symmetrify_full(bls_ctx* ctx, int dtype, int64_t nb, const int64_t* blocksizes, const int64_t* it_colptr,
                        const int64_t* it_rowval, const int64_t* it_nzval, const void* data, const int64_t* blocks,
                        int64_t nblocks, void* mat, int64_t m) {
  BLS_GUARD({
    if (!ctx || nb < 0 || (nb > 0 && (!blocksizes || !it_colptr))) throw Error(BLS_EINVAL, "null argument");
    if (dtype != BLS_F64 && dtype != BLS_F32) throw Error(BLS_EINVAL, "unknown dtype");
    // the included blocks' sizes and 0-based starts in mat (-1: left out), as symmetrifyfull! forms them
    std::vector<int64_t> lengths((size_t)nb, 0), starts((size_t)nb, -1);
    if (!blocks) {
      int64_t cur = 0;
      for (int64_t b = 0; b < nb; ++b) {
        lengths[b] = blocksizes[b];
        starts[b] = cur;
        cur += blocksizes[b];
      }
    } else {
      if (nblocks < 0) throw Error(BLS_EINVAL, "nblocks is negative");
      if (nblocks == 0) {
        if (m != 0)
          throw Error(BLS_EDIM, "Target matrix has size (" + std::to_string(m) + ", " + std::to_string(m) + "), expected (0, 0)");
        return BLS_OK;
      }
      for (int64_t i = 0; i < nblocks; ++i)
        if (blocks[i] < 0 || blocks[i] >= nb)
          throw Error(BLS_EINVAL, "BoundsError: block " + std::to_string(blocks[i] + 1) + " of " + std::to_string(nb));
      for (int64_t i = 0; i < nblocks; ++i) {
        const int64_t b = blocks[i];
        if (lengths[b] != 0) throw Error(BLS_EINVAL, "Block " + std::to_string(b + 1) + " is listed more than once");
        lengths[b] = blocksizes[b];
      }
      int64_t cur = 0;
      for (int64_t i = 0; i < nblocks; ++i) {
        starts[blocks[i]] = cur;
        cur += blocksizes[blocks[i]];
      }
    }
    int64_t total = 0;
    for (int64_t b = 0; b < nb; ++b) total += lengths[b];
    if (m != total)
      throw Error(BLS_EDIM, "Target matrix has size (" + std::to_string(m) + ", " + std::to_string(m) + "), expected (" +
                                std::to_string(total) + ", " + std::to_string(total) + ")");
    // the blocks to copy, in indicestransposed's order; of (r, c) and (c, r) only the later one (it overwrites all the
    // earlier one wrote)
    std::vector<SymBlock> list;
    std::vector<std::pair<int64_t, int64_t>> rc;
    for (int64_t r = 0; r < nb; ++r)
      for (int64_t k = it_colptr[r]; k < it_colptr[r + 1]; ++k) {
        const int64_t c = it_rowval[k];
        if (c < 0 || c >= nb) throw Error(BLS_EINVAL, "indicestransposed names a block column out of range");
        if (starts[c] < 0 || starts[r] < 0) continue;
        list.push_back(SymBlock{it_nzval[k], starts[r], starts[c], (int32_t)lengths[r], (int32_t)lengths[c], r == c ? 1 : 0, 0});
        rc.emplace_back(r, c);
      }
    std::map<std::pair<int64_t, int64_t>, size_t> last;
    for (size_t i = 0; i < rc.size(); ++i) last[rc[i]] = i;
    std::vector<SymBlock> keep;
    keep.reserve(list.size());
    for (size_t i = 0; i < list.size(); ++i) {
      if (!list[i].diag) {
        const auto it = last.find({rc[i].second, rc[i].first});
        if (it != last.end() && it->second > i) continue;
      }
      keep.push_back(list[i]);
    }
    if ((m > 0 && !mat) || (!keep.empty() && !data)) throw Error(BLS_EINVAL, "null argument");
    launch_symmetrify(ctx->stream, dtype, data, keep.data(), (int64_t)keep.size(), mat, m);
    return BLS_OK;
  })
}

}  // extern "C"
