// Host-side layout of an elimination: the integer structure, the reduced system's block pattern, the R -> S map and
// the CSC scatter map. These are the reference's setup steps (run once per structure), restated 0-based and organised
// for million-point scenes: couplings are bucketed by counting sort, and the pattern is built per block column from
// the column's own couplings in parallel, with no global list of pairs.
//
// Reference: src/schur_description.jl:16-101 (description), src/schur_structure.jl:70-166 (layout), :204-228
// (ordering), :241-323 (pattern), :406-431 (R -> S map), src/schur_reduction.jl:30-92 (workspace index and column
// chunks), src/SparseBlockLinearSystem.jl:43-64, 233-282 (retained storage, scatter map).
#include "host_layout.hpp"

#include <algorithm>
#include <map>
#include <cstring>
#include <limits>
#include <numeric>
#include <omp.h>

namespace bls {

static void check_dim(int64_t d, int64_t i) {
  if (d < 1 || d > 65535)
    throw Error(BLS_EINVAL, "Block " + std::to_string(i + 1) + " has dimension " + std::to_string(d) +
                                "; dimensions must be between 1 and 65535");
}

// Column chunks of equal work, couplings plus the diagonal (src/schur_reduction.jl:30-49). The target is compared in
// double, as the reference compares an Int against (total * k) / K.
std::vector<int64_t> partition_columns(const std::vector<int64_t>& retained_ptr, int64_t K) {
  const int64_t n = (int64_t)retained_ptr.size() - 1;
  const int64_t total = retained_ptr[n] - retained_ptr[0] + n;
  std::vector<int64_t> out;
  int64_t start = 0;   // 0-based first block of the next range
  for (int64_t k = 1; k <= K; ++k) {
    int64_t stop = start;   // exclusive
    if (k == K) {
      stop = n;
    } else {
      const double target = (double)(total * k) / (double)K;
      // the reference's `stop` is inclusive and 1-based; with s = exclusive 0-based stop the test on block s reads
      // retained_ptr[s + 1] - retained_ptr[0] + (s + 1) <= target
      while (stop < n && (double)(retained_ptr[stop + 1] - retained_ptr[0] + (stop + 1)) <= target) ++stop;
    }
    out.push_back(start);
    out.push_back(stop);
    start = stop;
  }
  return out;
}

void finish_structure(Structure& st, const std::vector<std::vector<int64_t>>& couplings) {
  const int64_t nrb = st.nrblocks, neb = st.neblocks;
  if ((int64_t)couplings.size() != neb) throw Error(BLS_EDIM, "Number of coupling lists must match the number of eliminated blocks");
  if (st.nchunks < 1) throw Error(BLS_EINVAL, "nchunks must be at least 1");
  if (st.min_work < 0) throw Error(BLS_EINVAL, "min_work must be non-negative");
  for (int64_t i = 0; i < nrb; ++i) check_dim(st.r_dims[i], i);
  for (int64_t i = 0; i < neb; ++i) check_dim(st.e_dims[i], i);
  {
    std::vector<int64_t> seen(nrb, -1);
    for (int64_t e = 0; e < neb; ++e)
      for (int64_t r : couplings[e]) {
        if (r < 0 || r >= nrb) throw Error(BLS_EINVAL, "Eliminated block " + std::to_string(e + 1) + " references retained block " + std::to_string(r + 1));
        if (seen[r] == e) throw Error(BLS_EINVAL, "Retained block " + std::to_string(r + 1) + " is listed more than once in the couplings of eliminated block " + std::to_string(e + 1));
        seen[r] = e;
      }
  }
  st.boffsets_r.resize(nrb);
  st.nr = 0;
  for (int64_t i = 0; i < nrb; ++i) { st.boffsets_r[i] = st.nr; st.nr += st.r_dims[i]; }
  st.boffsets_e.resize(neb);
  st.eoffsets.resize(neb);
  int64_t ne = 0, eo = 0;
  for (int64_t i = 0; i < neb; ++i) {
    st.boffsets_e[i] = ne; ne += st.e_dims[i];
    st.eoffsets[i] = eo; eo += st.e_dims[i] * st.e_dims[i];
  }
  st.ne = ne;
  st.E_length = eo;
  st.eliminated_ptr.assign(neb + 1, 0);
  for (int64_t e = 0; e < neb; ++e) st.eliminated_ptr[e + 1] = st.eliminated_ptr[e] + (int64_t)couplings[e].size();
  const int64_t nc = st.eliminated_ptr[neb];
  st.entry_retained.resize(nc);
  st.coffsets.resize(nc);
  int64_t coff = 0;
  st.max_coupled_dim = 0;
  for (int64_t e = 0; e < neb; ++e) {
    int64_t* er = st.entry_retained.data() + st.eliminated_ptr[e];
    std::copy(couplings[e].begin(), couplings[e].end(), er);
    std::sort(er, er + couplings[e].size());
    int64_t obs_dim = 0;
    for (size_t i = 0; i < couplings[e].size(); ++i) {
      st.coffsets[st.eliminated_ptr[e] + (int64_t)i] = coff;
      coff += st.r_dims[er[i]] * st.e_dims[e];
      obs_dim += st.r_dims[er[i]];
    }
    st.max_coupled_dim = std::max(st.max_coupled_dim, obs_dim);
  }
  st.C_length = coff;
  // runs of e_dims and their chunks (src/schur_structure.jl:138-150)
  st.e_run_first.clear();
  for (int64_t e = 0; e < neb; ++e)
    if (e == 0 || st.e_dims[e] != st.e_dims[e - 1]) st.e_run_first.push_back(e);
  st.e_run_first.push_back(neb);
  st.chunks.clear();
  for (size_t g = 0; g + 1 < st.e_run_first.size(); ++g) {
    const int64_t first = st.e_run_first[g], len = st.e_run_first[g + 1] - first;
    const int64_t sz = (len + st.nchunks - 1) / st.nchunks;
    for (int64_t k = 0; k < st.nchunks; ++k) {
      int64_t a = first + k * sz, b = std::min(first + len, a + sz);
      if (b < a) b = a;   // an empty range starts where the reference's does
      st.chunks.push_back(a);
      st.chunks.push_back(b);
    }
  }
  // workspace index (src/schur_reduction.jl:71-85): camera-major couplings, ascending coupling index per camera
  st.entry_eliminated.resize(nc);
  st.retained_ptr.assign(nrb + 1, 0);
  for (int64_t e = 0; e < neb; ++e)
    for (int64_t c = st.eliminated_ptr[e]; c < st.eliminated_ptr[e + 1]; ++c) {
      st.entry_eliminated[c] = e;
      st.retained_ptr[st.entry_retained[c] + 1] += 1;
    }
  for (int64_t r = 0; r < nrb; ++r) st.retained_ptr[r + 1] += st.retained_ptr[r];
  st.retained_entry.resize(nc);
  std::vector<int64_t> pos(st.retained_ptr.begin(), st.retained_ptr.end() - 1);
  for (int64_t c = 0; c < nc; ++c) st.retained_entry[pos[st.entry_retained[c]]++] = c;
  st.col_chunks = partition_columns(st.retained_ptr, std::max<int64_t>(st.nchunks, 1));
  // retained pairs: sorted, unique, validated (src/schur_structure.jl:155-158)
  std::sort(st.retained_pairs.begin(), st.retained_pairs.end());
  for (auto& p : st.retained_pairs)
    if (!(0 <= p.first && p.first < p.second && p.second < nrb)) throw Error(BLS_EINVAL, "Retained pair must satisfy i < j within the retained blocks");
  st.retained_pairs.erase(std::unique(st.retained_pairs.begin(), st.retained_pairs.end()), st.retained_pairs.end());
}

Structure structure_positional(const std::vector<int64_t>& r_dims, const std::vector<int64_t>& e_dims,
                               const std::vector<std::vector<int64_t>>& couplings, int64_t nchunks, int64_t min_work) {
  Structure st;
  st.nrblocks = (int64_t)r_dims.size();
  st.neblocks = (int64_t)e_dims.size();
  st.r_dims = r_dims;
  st.e_dims = e_dims;
  st.nchunks = nchunks;
  st.min_work = min_work;
  st.order.resize(st.nrblocks + st.neblocks);
  std::iota(st.order.begin(), st.order.end(), 0);
  finish_structure(st, couplings);
  return st;
}

Structure structure_from_description(int64_t n, const int64_t* blocksizes, int64_t K, const int64_t* rb_ptr,
                                     const int64_t* rb_idx, const uint8_t* eliminated, int64_t nchunks, int64_t min_work,
                                     const int64_t* rowblocksizes) {
  for (int64_t i = 0; i < n; ++i) check_dim(blocksizes[i], i);
  int64_t nret = 0;
  for (int64_t i = 0; i < n; ++i) nret += eliminated[i] ? 0 : 1;
  if (!(nret > 0 && nret < n))
    throw Error(BLS_EINVAL, "An elimination needs at least one retained and one eliminated column block; got " +
                                std::to_string(nret) + " retained and " + std::to_string(n - nret) + " eliminated");
  // one pass over the row blocks (src/schur_description.jl:37-59); coupled (e, r) pairs bucketed by e afterwards
  std::vector<int64_t> seen(n, -1), cnt(n + 1, 0);
  std::vector<char> hasrow(rowblocksizes ? n : 0, 0);
  for (int64_t k = 0; k < K; ++k) {
    if (rowblocksizes && rowblocksizes[k] < 1)
      throw Error(BLS_EINVAL, "Row block " + std::to_string(k + 1) + " has " + std::to_string(rowblocksizes[k]) + " rows; every row block needs at least 1 row");
    int64_t e = -1;
    for (int64_t p = rb_ptr[k]; p < rb_ptr[k + 1]; ++p) {
      const int64_t b = rb_idx[p];
      if (b < 0 || b >= n) throw Error(BLS_EINVAL, "Row block " + std::to_string(k + 1) + " touches column block " + std::to_string(b + 1) + ", but there are " + std::to_string(n) + " column blocks");
      if (seen[b] == k) throw Error(BLS_EINVAL, "Row block " + std::to_string(k + 1) + " lists column block " + std::to_string(b + 1) + " more than once");
      seen[b] = k;
      if (rowblocksizes) hasrow[b] = 1;
      if (eliminated[b]) {
        if (e >= 0) throw Error(BLS_EINVAL, "Row block " + std::to_string(k + 1) + " touches two eliminated column blocks, " + std::to_string(e + 1) + " and " + std::to_string(b + 1) + "; a row block may touch at most one");
        e = b;
      }
    }
    if (e >= 0)
      for (int64_t p = rb_ptr[k]; p < rb_ptr[k + 1]; ++p)
        if (!eliminated[rb_idx[p]]) cnt[e + 1] += 1;
  }
  if (rowblocksizes)
    for (int64_t b = 0; b < n; ++b)
      if (eliminated[b] && !hasrow[b]) throw Error(BLS_EINVAL, "Eliminated column block " + std::to_string(b + 1) + " is in no row block; eliminating a block needs at least one row");
  for (int64_t b = 0; b < n; ++b) cnt[b + 1] += cnt[b];
  std::vector<int64_t> coupled(cnt[n]);
  {
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t k = 0; k < K; ++k) {
      int64_t e = -1;
      for (int64_t p = rb_ptr[k]; p < rb_ptr[k + 1]; ++p)
        if (eliminated[rb_idx[p]]) e = rb_idx[p];
      if (e >= 0)
        for (int64_t p = rb_ptr[k]; p < rb_ptr[k + 1]; ++p)
          if (!eliminated[rb_idx[p]]) coupled[fill[e]++] = rb_idx[p];
    }
  }
  // unique!(sort!(coupled[b])) per eliminated block; keep the unique length per block
  std::vector<int64_t> ulen(n, 0), rmin(n, std::numeric_limits<int64_t>::max());
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < n; ++b) {
    int64_t* a = coupled.data() + cnt[b];
    int64_t* z = coupled.data() + cnt[b + 1];
    std::sort(a, z);
    ulen[b] = std::unique(a, z) - a;
    if (ulen[b] > 0) rmin[b] = a[0];
  }
  // layout order (sort_schur_blocks): retained by size descending, eliminated by (size descending, smallest coupled
  // retained block in the caller's numbering); stable, as Julia's default sort
  std::vector<int64_t> order;
  order.reserve(n);
  for (int64_t i = 0; i < n; ++i) if (!eliminated[i]) order.push_back(i);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return blocksizes[a] > blocksizes[b]; });
  std::vector<int64_t> eorder;
  eorder.reserve(n - nret);
  for (int64_t i = 0; i < n; ++i) if (eliminated[i]) eorder.push_back(i);
  std::stable_sort(eorder.begin(), eorder.end(), [&](int64_t a, int64_t b) {
    if (blocksizes[a] != blocksizes[b]) return blocksizes[a] > blocksizes[b];
    return rmin[a] < rmin[b];
  });
  order.insert(order.end(), eorder.begin(), eorder.end());
  std::vector<int64_t> position(n);
  for (int64_t p = 0; p < n; ++p) position[order[p]] = p;
  std::vector<std::vector<int64_t>> couplings(n - nret);
  for (int64_t p = nret; p < n; ++p) {
    const int64_t b = order[p];
    auto& c = couplings[p - nret];
    c.resize(ulen[b]);
    for (int64_t i = 0; i < ulen[b]; ++i) c[i] = position[coupled[cnt[b] + i]];
    std::sort(c.begin(), c.end());
  }
  Structure st;
  st.nrblocks = nret;
  st.neblocks = n - nret;
  st.r_dims.resize(nret);
  st.e_dims.resize(n - nret);
  for (int64_t p = 0; p < nret; ++p) st.r_dims[p] = blocksizes[order[p]];
  for (int64_t p = nret; p < n; ++p) st.e_dims[p - nret] = blocksizes[order[p]];
  // pairs of retained blocks sharing a row block (src/schur_description.jl:76-87), layout numbering
  std::vector<int64_t> rs;
  for (int64_t k = 0; k < K; ++k) {
    rs.clear();
    for (int64_t p = rb_ptr[k]; p < rb_ptr[k + 1]; ++p)
      if (!eliminated[rb_idx[p]]) rs.push_back(position[rb_idx[p]]);
    for (size_t a = 1; a < rs.size(); ++a)
      for (size_t c = 0; c < a; ++c) st.retained_pairs.push_back({std::min(rs[a], rs[c]), std::max(rs[a], rs[c])});
  }
  st.order = order;
  st.nchunks = nchunks;
  st.min_work = min_work;
  finish_structure(st, couplings);
  return st;
}

// build_schur_pattern (src/schur_structure.jl:241-323). Column r2 of the block pattern holds r2 itself, every r1 <= r2
// sharing an eliminated block with r2 (found from r2's couplings: for coupling c2 of point e, every c1 <= c2 of e),
// the retained pairs and the extra pairs. Columns are independent, so they are built in parallel.
Pattern build_pattern(const Structure& st, const std::vector<std::pair<int64_t, int64_t>>& extra) {
  const int64_t nrb = st.nrblocks;
  Pattern P;
  std::vector<std::vector<int64_t>> add(nrb);
  for (auto& p : st.retained_pairs) add[p.second].push_back(p.first);
  for (auto& p : extra) {
    if (p.first < 0 || p.first >= nrb || p.second < 0 || p.second >= nrb)
      throw Error(BLS_EINVAL, "Extra block pair (" + std::to_string(p.first + 1) + ", " + std::to_string(p.second + 1) + ") is outside the " + std::to_string(nrb) + " retained blocks");
    add[std::max(p.first, p.second)].push_back(std::min(p.first, p.second));
  }
  std::vector<std::vector<int32_t>> cols(nrb);
#pragma omp parallel
  {
    std::vector<int64_t> mark(nrb, -1);
    std::vector<int32_t> rows;
#pragma omp for schedule(dynamic, 16)
    for (int64_t r2 = 0; r2 < nrb; ++r2) {
      rows.clear();
      auto take = [&](int64_t r1) { if (mark[r1] != r2) { mark[r1] = r2; rows.push_back((int32_t)r1); } };
      take(r2);
      for (int64_t q = st.retained_ptr[r2]; q < st.retained_ptr[r2 + 1]; ++q) {
        const int64_t c2 = st.retained_entry[q], e = st.entry_eliminated[c2];
        for (int64_t c1 = st.eliminated_ptr[e]; c1 <= c2; ++c1) take(st.entry_retained[c1]);
      }
      for (int64_t r1 : add[r2]) take(r1);
      std::sort(rows.begin(), rows.end());
      cols[r2] = rows;
    }
  }
  P.block_colptr.assign(nrb + 1, 0);
  for (int64_t c = 0; c < nrb; ++c) P.block_colptr[c + 1] = P.block_colptr[c] + (int64_t)cols[c].size();
  const int64_t nb = P.block_colptr[nrb];
  P.block_rowval.resize(nb);
  P.block_row_offsets.resize(nb);
  P.col_heights.resize(nrb);
  for (int64_t c = 0; c < nrb; ++c) {
    int64_t h = 0;
    for (size_t i = 0; i < cols[c].size(); ++i) {
      const int64_t k = P.block_colptr[c] + (int64_t)i;
      P.block_rowval[k] = cols[c][i];
      P.block_row_offsets[k] = h;
      h += st.r_dims[cols[c][i]];
    }
    P.col_heights[c] = h;
  }
  // scalar CSC: each scalar column of block column r2 lists the rows of its blocks in block order (already sorted)
  P.S_colptr.assign(st.nr + 1, 0);
  for (int64_t r2 = 0; r2 < nrb; ++r2)
    for (int64_t w = 0; w < st.r_dims[r2]; ++w) {
      const int64_t j = st.boffsets_r[r2] + w;
      P.S_colptr[j + 1] = P.S_colptr[j] + P.col_heights[r2];
    }
  P.S_rowval.resize(P.S_colptr[st.nr]);
  P.diag_inds.resize(st.nr);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    for (int64_t w = 0; w < st.r_dims[r2]; ++w) {
      const int64_t j = st.boffsets_r[r2] + w;
      int64_t q = P.S_colptr[j];
      for (int64_t k = P.block_colptr[r2]; k < P.block_colptr[r2 + 1]; ++k) {
        const int64_t r1 = P.block_rowval[k];
        if (r1 == r2) P.diag_inds[j] = q + w;
        for (int64_t a = 0; a < st.r_dims[r1]; ++a) P.S_rowval[q++] = st.boffsets_r[r1] + a;
      }
    }
  }
  // retained storage on the pattern (TransposedPattern of the block pattern): block (row r2, column r1) of R, for the
  // k-th block of column r2, starts after the blocks of the previous rows, d_r2 x d_r1 column-major
  P.R_block_start.resize(nb);
  int64_t start = 0;
  for (int64_t r2 = 0; r2 < nrb; ++r2)
    for (int64_t k = P.block_colptr[r2]; k < P.block_colptr[r2 + 1]; ++k) {
      P.R_block_start[k] = start;
      start += st.r_dims[r2] * st.r_dims[P.block_rowval[k]];
    }
  P.R_length = start;
  return P;
}

// build_r_to_s_map, block-level (src/schur_structure.jl:406-431), for R laid out on the pattern: R block (r2, r1)
// maps onto S block (r1, r2); a diagonal block maps its upper triangle only (-1 elsewhere).
std::vector<int64_t> build_r_to_s(const Structure& st, const Pattern& P) {
  std::vector<int64_t> m(P.R_length, -1);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t r2 = 0; r2 < st.nrblocks; ++r2) {
    const int64_t drow = st.r_dims[r2], stride = P.col_heights[r2];
    for (int64_t k = P.block_colptr[r2]; k < P.block_colptr[r2 + 1]; ++k) {
      const int64_t r1 = P.block_rowval[k], dcol = st.r_dims[r1];
      const int64_t base = P.S_colptr[st.boffsets_r[r2]] + P.block_row_offsets[k];
      const int64_t ds = P.R_block_start[k];
      if (r1 == r2) {
        for (int64_t col = 0; col < dcol; ++col)
          for (int64_t row = 0; row <= col; ++row) m[ds + col * drow + row] = base + col * stride + row;
      } else {
        for (int64_t col = 0; col < dcol; ++col)
          for (int64_t row = 0; row < drow; ++row) m[ds + col * drow + row] = base + row * stride + col;
      }
    }
  }
  return m;
}

// makesparseindices (src/SparseBlockLinearSystem.jl:233-282) for R on the pattern. Scalar column j of R's block
// column b: with symmetrify, first the transposes of the blocks (b, r1 < b) — R's blocks in row b, i.e. the pattern's
// column b without its diagonal — then the blocks (r, b) for r >= b, in ascending r.
int64_t sparse_indices(const Structure& st, const Pattern& P, bool symmetric, int64_t* colptr, int64_t* rowval, int64_t* map) {
  const int64_t nrb = st.nrblocks;
  // R's block columns: block (r, b), r >= b, is the pattern's block (b, r) of column r
  std::vector<int64_t> lptr(nrb + 1, 0);
  for (int64_t r = 0; r < nrb; ++r)
    for (int64_t k = P.block_colptr[r]; k < P.block_colptr[r + 1]; ++k) lptr[P.block_rowval[k] + 1] += 1;
  for (int64_t b = 0; b < nrb; ++b) lptr[b + 1] += lptr[b];
  std::vector<int64_t> lrow(lptr[nrb]), lk(lptr[nrb]);
  {
    std::vector<int64_t> fill(lptr.begin(), lptr.end() - 1);
    for (int64_t r = 0; r < nrb; ++r)
      for (int64_t k = P.block_colptr[r]; k < P.block_colptr[r + 1]; ++k) {
        const int64_t b = P.block_rowval[k];
        lrow[fill[b]] = r;
        lk[fill[b]++] = k;
      }
  }
  int64_t diagspace = 0;
  for (int64_t b = 0; b < nrb; ++b)
    if (lptr[b + 1] > lptr[b] && lrow[lptr[b]] == b) diagspace += st.r_dims[b] * st.r_dims[b];
  const int64_t nnz = symmetric ? 2 * P.R_length - diagspace : P.R_length;
  if (!colptr && !rowval && !map) return nnz;
  int64_t ind = 0, col = 0;
  if (colptr) colptr[0] = 0;
  for (int64_t b = 0; b < nrb; ++b) {
    const int64_t cb = st.r_dims[b];
    const bool has_diag = lptr[b + 1] > lptr[b] && lrow[lptr[b]] == b;
    const int64_t up_end = symmetric ? P.block_colptr[b + 1] - (has_diag ? 1 : 0) : P.block_colptr[b];
    for (int64_t inner = 0; inner < cb; ++inner) {
      for (int64_t k = P.block_colptr[b]; k < up_end; ++k) {
        const int64_t r = P.block_rowval[k], s = st.boffsets_r[r], c = st.r_dims[r];
        int64_t v = P.R_block_start[k] + inner;
        for (int64_t i = 0; i < c; ++i) {
          if (rowval) rowval[ind] = s + i;
          if (map) map[ind] = v;
          ++ind;
          v += cb;
        }
      }
      for (int64_t q = lptr[b]; q < lptr[b + 1]; ++q) {
        const int64_t r = lrow[q], s = st.boffsets_r[r], c = st.r_dims[r];
        const int64_t v = P.R_block_start[lk[q]] + inner * c;
        for (int64_t i = 0; i < c; ++i) {
          if (rowval) rowval[ind] = s + i;
          if (map) map[ind] = v + i;
          ++ind;
        }
      }
      ++col;
      if (colptr) colptr[col] = ind;
    }
  }
  return nnz;
}

}  // namespace bls

namespace bls {

// SchurJacobianStructure(structure, e_rows; free_rows, free_retained, nchunks) (src/schur_jacobian.jl:59-160)
QRStructure qr_structure(const Structure& st, const std::vector<int64_t>& e_rows, const std::vector<int64_t>& free_rows,
                         const std::vector<std::vector<int64_t>>& free_retained, int64_t nchunks) {
  QRStructure q;
  q.schur = st;
  const int64_t ne = st.neblocks, nrb = st.nrblocks, nfree = (int64_t)free_rows.size();
  if ((int64_t)e_rows.size() != ne) throw Error(BLS_EDIM, "Number of eliminated row counts (" + std::to_string(e_rows.size()) + ") must match the number of eliminated blocks (" + std::to_string(ne) + ")");
  if ((int64_t)free_retained.size() != nfree) throw Error(BLS_EDIM, "Number of free groups' retained lists must match the number of free row counts");
  if (nchunks < 1) throw Error(BLS_EINVAL, "nchunks must be at least 1, got " + std::to_string(nchunks));
  for (int64_t e = 0; e < ne; ++e)
    if (e_rows[e] < 1) throw Error(BLS_EINVAL, "Eliminated block " + std::to_string(e + 1) + " has " + std::to_string(e_rows[e]) + " rows; every eliminated block needs at least 1 row");
  for (int64_t g = 0; g < nfree; ++g)
    if (free_rows[g] < 1) throw Error(BLS_EINVAL, "Free group " + std::to_string(g + 1) + " has " + std::to_string(free_rows[g]) + " rows; every free group needs at least 1 row");
  {
    std::vector<int64_t> seen(nrb, -1);
    for (int64_t g = 0; g < nfree; ++g)
      for (int64_t r : free_retained[g]) {
        if (r < 0 || r >= nrb) throw Error(BLS_EINVAL, "Free group " + std::to_string(g + 1) + " references retained block " + std::to_string(r + 1));
        if (seen[r] == g) throw Error(BLS_EINVAL, "Retained block " + std::to_string(r + 1) + " is listed more than once in free group " + std::to_string(g + 1));
        seen[r] = g;
      }
  }
  const int64_t nt = ne + nfree;
  q.ntables = nt;
  q.e_rows = e_rows;
  q.free_rows = free_rows;
  q.table_nrows.resize(nt); q.table_ncols.resize(nt); q.table_top.resize(nt); q.table_ptr.assign(nt + 1, 0);
  for (int64_t t = 0; t < nt; ++t) {
    std::vector<int64_t> rs;
    if (t < ne) rs.assign(st.entry_retained.begin() + st.eliminated_ptr[t], st.entry_retained.begin() + st.eliminated_ptr[t + 1]);
    else { rs = free_retained[t - ne]; std::sort(rs.begin(), rs.end()); }
    int64_t col = 0;
    for (int64_t r : rs) {
      q.entry_retained.push_back(r);
      q.entry_col.push_back(col);
      q.entry_table.push_back(t);
      col += st.r_dims[r];
    }
    q.table_ptr[t + 1] = (int64_t)q.entry_retained.size();
    const int64_t de = t < ne ? st.e_dims[t] : 0;
    q.table_top[t] = de;
    q.table_nrows[t] = t < ne ? e_rows[t] + de : free_rows[t - ne];
    q.table_ncols[t] = col + de + 1;
  }
  q.table_offsets.assign(nt + 1, 0); q.raw_offsets.assign(nt + 1, 0); q.residual_offsets.assign(nt + 1, 0); q.reduced_offsets.assign(nt + 1, 0);
  for (int64_t t = 0; t < nt; ++t) {
    q.table_offsets[t + 1] = q.table_offsets[t] + q.table_nrows[t] * q.table_ncols[t];
    q.raw_offsets[t + 1] = q.raw_offsets[t] + q.table_nrows[t] * (q.table_ncols[t] - 1);
    q.residual_offsets[t + 1] = q.residual_offsets[t] + q.table_nrows[t];
    q.reduced_offsets[t + 1] = q.reduced_offsets[t] + q.table_nrows[t] - q.table_top[t];
  }
  const int64_t nent = (int64_t)q.entry_retained.size();
  q.retained_ptr.assign(nrb + 1, 0);
  for (int64_t u = 0; u < nent; ++u) q.retained_ptr[q.entry_retained[u] + 1] += 1;
  for (int64_t r = 0; r < nrb; ++r) q.retained_ptr[r + 1] += q.retained_ptr[r];
  q.retained_entry.resize(nent);
  {
    std::vector<int64_t> pos(q.retained_ptr.begin(), q.retained_ptr.end() - 1);
    for (int64_t u = 0; u < nent; ++u) q.retained_entry[pos[q.entry_retained[u]]++] = u;
  }
  q.doffsets.assign(nrb + 1, 0);
  for (int64_t r = 0; r < nrb; ++r) q.doffsets[r + 1] = q.doffsets[r] + st.r_dims[r] * st.r_dims[r];
  q.col_chunks = partition_columns(q.retained_ptr, nchunks);
  return q;
}

// SchurJacobianStructure(blocksizes, rowblocks, rowblocksizes; eliminated) (src/schur_description.jl:137-189): each row
// block's rows go to its eliminated block's table, or to the table of its free group (row blocks with the same retained
// blocks, numbered by first appearance), in row-block order.
QRStructure qr_structure_from_description(int64_t n, const int64_t* blocksizes, int64_t K, const int64_t* rb_ptr, const int64_t* rb_idx,
                                          const int64_t* rowblocksizes, const uint8_t* eliminated, int64_t nchunks, int64_t min_work) {
  Structure st = structure_from_description(n, blocksizes, K, rb_ptr, rb_idx, eliminated, nchunks, min_work, rowblocksizes);
  const int64_t nret = st.nrblocks, ne = st.neblocks;
  std::vector<int64_t> position(n);
  for (int64_t p = 0; p < n; ++p) position[st.order[p]] = p;
  std::vector<int64_t> row_table(K), row_first(K), e_rows(ne, 0), free_rows_v, row_ptr(K + 1, 0), row_blocks(rb_ptr[K]);
  std::vector<std::vector<int64_t>> free_retained;
  std::map<std::vector<int64_t>, int64_t> group;
  for (int64_t k = 0; k < K; ++k) row_ptr[k + 1] = rb_ptr[k + 1] - rb_ptr[0];
  for (int64_t k = 0; k < K; ++k) {
    const int64_t m = rowblocksizes[k];
    int64_t e = -1;
    for (int64_t p = rb_ptr[k]; p < rb_ptr[k + 1]; ++p) {
      row_blocks[p - rb_ptr[0]] = position[rb_idx[p]];
      if (eliminated[rb_idx[p]]) e = rb_idx[p];
    }
    std::sort(row_blocks.begin() + row_ptr[k], row_blocks.begin() + row_ptr[k + 1]);
    if (e >= 0) {
      const int64_t t = position[e] - nret;
      row_table[k] = t;
      row_first[k] = e_rows[t];
      e_rows[t] += m;
    } else {
      std::vector<int64_t> rs(row_blocks.begin() + row_ptr[k], row_blocks.begin() + row_ptr[k + 1]);
      auto it = group.find(rs);
      int64_t g;
      if (it == group.end()) {
        free_retained.push_back(rs);
        free_rows_v.push_back(0);
        g = (int64_t)free_rows_v.size() - 1;
        group[rs] = g;
      } else {
        g = it->second;
      }
      row_table[k] = ne + g;
      row_first[k] = free_rows_v[g];
      free_rows_v[g] += m;
    }
  }
  QRStructure q = qr_structure(st, e_rows, free_rows_v, free_retained, nchunks);
  q.row_table = row_table;
  q.row_first = row_first;
  q.row_nrows.assign(rowblocksizes, rowblocksizes + K);
  q.row_ptr = row_ptr;
  q.row_blocks = row_blocks;
  return q;
}

}  // namespace bls
