// Oracle: a CPU restatement of BlockLinearSystems.jl v0.3.1's elimination path, used ONLY as the checker
// (tests, the smoke check) and as the timed CPU baseline of bench.py. Nothing in the product links or calls it.
//
// Each function cites the reference file:line it restates. The reference is Julia (1-based); this file keeps
// 1-based integers internally (the `V1` accessor) so that each loop reads like the Julia it restates, and converts to
// 0-based at the extern "C" boundary. Floating-point operation order per entry follows the reference; the file is
// compiled with -ffp-contract=off because Julia does not contract a*b+c into an FMA.
//
// Threading: the reference threads its chunk loops with Polyester (ext/PolyesterExt.jl:12-23) when
// `use_threads` (src/threading.jl:28) says so; here OpenMP runs the same chunks.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>
#include <atomic>
#include <omp.h>

using i64 = int64_t;

namespace {

// ------------------------------------------------------------------------------------------------------------------
// 1-based containers
// ------------------------------------------------------------------------------------------------------------------
template <class T>
struct V1 {
  std::vector<T> v;
  V1() = default;
  explicit V1(i64 n, T x = T()) : v((size_t)n, x) {}
  T& operator()(i64 i) { return v[(size_t)(i - 1)]; }
  const T& operator()(i64 i) const { return v[(size_t)(i - 1)]; }
  i64 len() const { return (i64)v.size(); }
  void push(T x) { v.push_back(x); }
  T& last() { return v.back(); }
};
using IV = V1<i64>;

struct Range { i64 first, last; };   // Julia first:last (empty when last < first)

struct BlsError : std::runtime_error {
  int code;
  BlsError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
enum { ORC_OK = 0, ORC_NOT_PD = 1, ORC_EINVAL = -1, ORC_EDIM = -2, ORC_EPATTERN = -3 };

[[noreturn]] void arg_error(const std::string& m) { throw BlsError(ORC_EINVAL, m); }
[[noreturn]] void dim_error(const std::string& m) { throw BlsError(ORC_EDIM, m); }

// ------------------------------------------------------------------------------------------------------------------
// BlockRLE runs (src/BlockRLE.jl:3-29, 58-75, 170-177): runs of equal block sizes, adjacent equal runs merged
// ------------------------------------------------------------------------------------------------------------------
struct Runs {
  std::vector<i64> len, size;
  i64 nruns() const { return (i64)len.size(); }
  // runblockrange(rle, k) (src/BlockRLE.jl:174-177)
  Range blockrange(i64 k) const {
    i64 first = 1;
    for (i64 i = 1; i < k; ++i) first += len[i - 1];
    return {first, first + len[k - 1] - 1};
  }
};
Runs encode_runs(const IV& dims) {
  Runs r;
  for (i64 i = 1; i <= dims.len(); ++i) {
    i64 d = dims(i);
    if (!r.size.empty() && r.size.back() == d) r.len.back() += 1;
    else { r.len.push_back(1); r.size.push_back(d); }
  }
  return r;
}
void check_block_dim(i64 d, i64 i) {   // src/BlockRLE.jl:40-45
  if (!(1 <= d && d <= 65535)) arg_error("Block " + std::to_string(i) + " has dimension " + std::to_string(d) + "; dimensions must be between 1 and 65535");
}

// computestartindices (src/BlockRLE.jl:184-199)
IV start_indices(const IV& dims) {
  IV s(dims.len());
  i64 curr = 1;
  for (i64 i = 1; i <= dims.len(); ++i) { s(i) = curr; curr += dims(i); }
  return s;
}

// ------------------------------------------------------------------------------------------------------------------
// SchurStructure (src/schur_structure.jl:50-166)
// ------------------------------------------------------------------------------------------------------------------
struct Structure {
  i64 nr = 0, nrblocks = 0, neblocks = 0;
  IV r_dims, e_dims;
  Runs e_runs;
  IV boffsets_r, boffsets_e, eoffsets, eliminated_ptr, entry_retained, coffsets;
  i64 max_coupled_dim = 0;
  std::vector<std::vector<Range>> chunks;   // chunks[run][chunk]
  IV order;
  std::vector<std::pair<i64, i64>> retained_pairs;
  i64 nchunks = 1, min_work = 4096;
  // Jacobian-path description data (src/schur_description.jl:148-187); empty for a positional structure
  IV position, rowblock_eliminated;
};

// positional constructor (src/schur_structure.jl:70-166)
Structure make_structure(const IV& r_dims, const IV& e_dims, const std::vector<IV>& couplings, i64 nchunks, i64 min_work,
                         const IV* order, std::vector<std::pair<i64, i64>> retained_pairs) {
  Structure st;
  i64 nrblocks = r_dims.len(), neblocks = e_dims.len();
  if ((i64)couplings.size() != neblocks) dim_error("Number of coupling lists must match the number of eliminated blocks");
  if (nchunks < 1) arg_error("nchunks must be at least 1");
  if (min_work < 0) arg_error("min_work must be non-negative");
  for (i64 i = 1; i <= nrblocks; ++i) check_block_dim(r_dims(i), i);
  for (i64 i = 1; i <= neblocks; ++i) check_block_dim(e_dims(i), i);
  IV seen(nrblocks, 0);   // :89-96
  for (i64 e = 1; e <= neblocks; ++e) {
    for (i64 r : couplings[e - 1].v) {
      if (!(1 <= r && r <= nrblocks)) arg_error("Eliminated block " + std::to_string(e) + " references retained block " + std::to_string(r));
      if (seen(r) == e) arg_error("Retained block " + std::to_string(r) + " is listed more than once in the couplings of eliminated block " + std::to_string(e));
      seen(r) = e;
    }
  }
  st.nrblocks = nrblocks; st.neblocks = neblocks;
  st.r_dims = r_dims; st.e_dims = e_dims;
  st.e_runs = encode_runs(e_dims);
  st.nr = 0; for (i64 i = 1; i <= nrblocks; ++i) st.nr += r_dims(i);   // :98
  st.boffsets_r = start_indices(r_dims);                                 // :99
  st.boffsets_e = start_indices(e_dims);                                 // :100
  st.eoffsets = IV(neblocks);                                            // :102-108
  if (neblocks > 0) {
    st.eoffsets(1) = 1;
    for (i64 i = 2; i <= neblocks; ++i) st.eoffsets(i) = st.eoffsets(i - 1) + e_dims(i - 1) * e_dims(i - 1);
  }
  st.eliminated_ptr = IV(neblocks + 1);                                  // :110-115
  st.eliminated_ptr(1) = 1;
  for (i64 e = 1; e <= neblocks; ++e) st.eliminated_ptr(e + 1) = st.eliminated_ptr(e) + couplings[e - 1].len();
  i64 num_couplings = st.eliminated_ptr(neblocks + 1) - 1;
  st.entry_retained = IV(num_couplings);                                 // :117-130
  st.coffsets = IV(num_couplings);
  i64 curr_c_off = 1, idx = 1;
  for (i64 e = 1; e <= neblocks; ++e) {
    i64 de = e_dims(e);
    std::vector<i64> sorted_retained = couplings[e - 1].v;
    std::sort(sorted_retained.begin(), sorted_retained.end());
    for (i64 r : sorted_retained) {
      st.entry_retained(idx) = r;
      st.coffsets(idx) = curr_c_off;
      curr_c_off += r_dims(r) * de;
      idx += 1;
    }
  }
  st.max_coupled_dim = 0;                                                // :132-136
  for (i64 e = 1; e <= neblocks; ++e) {
    i64 obs_dim = 0;
    for (i64 r : couplings[e - 1].v) obs_dim += r_dims(r);
    st.max_coupled_dim = std::max(st.max_coupled_dim, obs_dim);
  }
  st.chunks.resize(st.e_runs.nruns());                                   // :138-150
  for (i64 g = 1; g <= st.e_runs.nruns(); ++g) {
    Range grp = st.e_runs.blockrange(g);
    i64 len = grp.last - grp.first + 1;
    i64 chunk_sz = (len + nchunks - 1) / nchunks;   // cld
    std::vector<Range> group_chunks((size_t)nchunks);
    for (i64 k = 1; k <= nchunks; ++k) {
      i64 first_idx = grp.first + (k - 1) * chunk_sz;
      i64 last_idx = std::min(grp.last, first_idx + chunk_sz - 1);
      group_chunks[k - 1] = first_idx <= last_idx ? Range{first_idx, last_idx} : Range{first_idx, first_idx - 1};
    }
    st.chunks[g - 1] = group_chunks;
  }
  i64 ntotal = nrblocks + neblocks;                                      // :152-158
  if (order) {
    if (order->len() != ntotal) dim_error("order has the wrong length");
    st.order = *order;
  } else {
    st.order = IV(ntotal);
    for (i64 i = 1; i <= ntotal; ++i) st.order(i) = i;
  }
  std::sort(retained_pairs.begin(), retained_pairs.end());
  for (auto& p : retained_pairs)
    if (!(1 <= p.first && p.first < p.second && p.second <= nrblocks)) arg_error("Retained pair must satisfy 1 <= i < j <= nrblocks");
  retained_pairs.erase(std::unique(retained_pairs.begin(), retained_pairs.end()), retained_pairs.end());   // unique!
  st.retained_pairs = retained_pairs;
  st.nchunks = nchunks; st.min_work = min_work;
  return st;
}

// sort_schur_blocks (src/schur_structure.jl:204-228). Julia 1.10's default sort is stable, so ties keep index order.
IV sort_schur_blocks(const std::vector<bool>& is_elim, const IV& sizes, const std::vector<std::vector<i64>>& coupled) {
  i64 n = (i64)is_elim.size();
  std::vector<i64> r_idx, e_idx;
  for (i64 i = 1; i <= n; ++i) (is_elim[i - 1] ? e_idx : r_idx).push_back(i);
  std::stable_sort(r_idx.begin(), r_idx.end(), [&](i64 a, i64 b) { return -sizes(a) < -sizes(b); });
  auto key = [&](i64 i) {
    const auto& c = coupled[i - 1];
    i64 r_min = c.empty() ? std::numeric_limits<i64>::max() : *std::min_element(c.begin(), c.end());
    return std::make_pair(-sizes(i), r_min);
  };
  std::stable_sort(e_idx.begin(), e_idx.end(), [&](i64 a, i64 b) { return key(a) < key(b); });
  IV out;
  for (i64 i : r_idx) out.push(i);
  for (i64 i : e_idx) out.push(i);
  return out;
}

// expand_block_perm (src/schur_structure.jl:173-194)
IV expand_block_perm(const IV& perm, const IV& sizes) {
  i64 nb = sizes.len();
  if (perm.len() != nb) dim_error("block_perm has the wrong length");
  std::vector<bool> hit((size_t)nb, false);
  for (i64 b : perm.v) {
    if (b < 1 || b > nb || hit[b - 1]) arg_error("block_perm must be a permutation");
    hit[b - 1] = true;
  }
  i64 total = 0; for (i64 s : sizes.v) total += s;
  IV bo(nb);
  if (nb > 0) bo(1) = 1;
  for (i64 i = 2; i <= nb; ++i) bo(i) = bo(i - 1) + sizes(i - 1);
  IV sp(total);
  i64 cursor = 1;
  for (i64 b : perm.v) for (i64 j = 1; j <= sizes(b); ++j) { sp(cursor) = bo(b) + j - 1; cursor += 1; }
  return sp;
}

// describe_elimination + description_structure + SchurStructure(blocksizes, rowblocks; eliminated)
// (src/schur_description.jl:16-101)
Structure structure_from_description(const IV& blocksizes, const std::vector<std::vector<i64>>& rowblocks,
                                     const std::vector<bool>& eliminated, const IV* rowblocksizes, i64 nchunks, i64 min_work) {
  i64 n = blocksizes.len(), K = (i64)rowblocks.size();
  if ((i64)eliminated.size() != n) dim_error("eliminated has the wrong length");
  if (rowblocksizes && rowblocksizes->len() != K) dim_error("rowblocksizes has the wrong length");
  for (i64 i = 1; i <= n; ++i) check_block_dim(blocksizes(i), i);
  i64 nret = 0; for (bool b : eliminated) nret += !b;
  if (!(nret > 0 && nret < n)) arg_error("An elimination needs at least one retained and one eliminated column block");
  IV seen(n, 0), rowblock_eliminated(K, 0);
  std::vector<std::vector<i64>> coupled((size_t)n);
  std::vector<bool> hasrow((size_t)n, false);
  for (i64 k = 1; k <= K; ++k) {                                         // :37-59
    if (rowblocksizes && (*rowblocksizes)(k) < 1) arg_error("Row block " + std::to_string(k) + " needs at least 1 row");
    i64 e = 0;
    for (i64 b : rowblocks[k - 1]) {
      if (!(1 <= b && b <= n)) arg_error("Row block " + std::to_string(k) + " touches column block " + std::to_string(b));
      if (seen(b) == k) arg_error("Row block " + std::to_string(k) + " lists column block " + std::to_string(b) + " more than once");
      seen(b) = k;
      hasrow[b - 1] = true;
      if (eliminated[b - 1]) {
        if (e != 0) arg_error("Row block " + std::to_string(k) + " touches two eliminated column blocks");
        e = b;
      }
    }
    rowblock_eliminated(k) = e;
    if (e != 0) for (i64 b : rowblocks[k - 1]) if (!eliminated[b - 1]) coupled[e - 1].push_back(b);
  }
  if (rowblocksizes)                                                      // :60-64
    for (i64 b = 1; b <= n; ++b)
      if (eliminated[b - 1] && !hasrow[b - 1]) arg_error("Eliminated column block " + std::to_string(b) + " is in no row block");
  for (auto& c : coupled) { std::sort(c.begin(), c.end()); c.erase(std::unique(c.begin(), c.end()), c.end()); }
  IV order = sort_schur_blocks(eliminated, blocksizes, coupled);         // :71
  IV position(n);
  for (i64 p = 1; p <= n; ++p) position(order(p)) = p;                    // invperm
  std::vector<IV> couplings;                                              // :73
  for (i64 p = nret + 1; p <= n; ++p) {
    IV c;
    for (i64 r : coupled[order(p) - 1]) c.push(position(r));
    std::sort(c.v.begin(), c.v.end());
    couplings.push_back(c);
  }
  std::vector<std::pair<i64, i64>> pairs;                                 // :76-87
  std::vector<i64> rs;
  for (i64 k = 1; k <= K; ++k) {
    rs.clear();
    for (i64 b : rowblocks[k - 1]) if (!eliminated[b - 1]) rs.push_back(position(b));
    for (i64 a = 2; a <= (i64)rs.size(); ++a)
      for (i64 c = 1; c <= a - 1; ++c) pairs.push_back({std::min(rs[a - 1], rs[c - 1]), std::max(rs[a - 1], rs[c - 1])});
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  IV r_dims(nret), e_dims(n - nret);                                      // :91-95
  for (i64 p = 1; p <= nret; ++p) r_dims(p) = blocksizes(order(p));
  for (i64 p = nret + 1; p <= n; ++p) e_dims(p - nret) = blocksizes(order(p));
  Structure st = make_structure(r_dims, e_dims, couplings, nchunks, min_work, &order, pairs);
  st.position = position;
  st.rowblock_eliminated = rowblock_eliminated;
  return st;
}

// ------------------------------------------------------------------------------------------------------------------
// build_schur_pattern (src/schur_structure.jl:241-323)
// ------------------------------------------------------------------------------------------------------------------
struct Pattern {
  i64 nrblocks = 0, nr = 0;
  IV block_colptr, block_rowval, block_row_offsets, col_heights;
  IV S_colptr, S_rowval, diag_inds;
};

Pattern build_schur_pattern(const Structure& st, const std::vector<std::pair<i64, i64>>& extra) {
  Pattern P;
  i64 nrb = st.nrblocks;
  P.nrblocks = nrb; P.nr = st.nr;
  // I_cov/J_cov, then sparse(I, J, true, n, n, |): per column the sorted unique rows
  std::vector<std::vector<i64>> cols((size_t)nrb);
  for (i64 e = 1; e <= st.neblocks; ++e) {
    i64 c_start = st.eliminated_ptr(e), c_end = st.eliminated_ptr(e + 1) - 1;
    for (i64 idx2 = c_start; idx2 <= c_end; ++idx2) {
      i64 r2 = st.entry_retained(idx2);
      for (i64 idx1 = c_start; idx1 <= idx2; ++idx1) cols[r2 - 1].push_back(st.entry_retained(idx1));
    }
  }
  for (auto& p : st.retained_pairs) cols[p.second - 1].push_back(p.first);
  for (auto& p : extra) {
    if (!(1 <= p.first && p.first <= nrb && 1 <= p.second && p.second <= nrb)) arg_error("Extra block pair is outside the retained blocks");
    cols[std::max(p.first, p.second) - 1].push_back(std::min(p.first, p.second));
  }
  for (i64 r = 1; r <= nrb; ++r) cols[r - 1].push_back(r);
  P.block_colptr = IV(nrb + 1);
  P.block_colptr(1) = 1;
  for (i64 c = 1; c <= nrb; ++c) {
    auto& v = cols[c - 1];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    P.block_colptr(c + 1) = P.block_colptr(c) + (i64)v.size();
    for (i64 r : v) P.block_rowval.push(r);
  }
  i64 nnz_blocks = P.block_rowval.len();
  P.col_heights = IV(nrb, 0);                                             // :284-295
  P.block_row_offsets = IV(nnz_blocks, 0);
  for (i64 r2 = 1; r2 <= nrb; ++r2) {
    i64 h = 0;
    for (i64 idx = P.block_colptr(r2); idx <= P.block_colptr(r2 + 1) - 1; ++idx) {
      i64 r1 = P.block_rowval(idx);
      P.block_row_offsets(idx) = h;
      h += st.r_dims(r1);
    }
    P.col_heights(r2) = h;
  }
  // :297-309 scalar pattern. Within a scalar column of block column r2 the rows are the blocks' rows in ascending block
  // order, which is already sorted and unique, so `sparse` keeps them as listed.
  P.S_colptr = IV(st.nr + 1);
  P.S_colptr(1) = 1;
  for (i64 r2 = 1; r2 <= nrb; ++r2) {
    for (i64 r_col = 1; r_col <= st.r_dims(r2); ++r_col) {
      i64 j = st.boffsets_r(r2) + r_col - 1;
      P.S_colptr(j + 1) = P.S_colptr(j) + P.col_heights(r2);
      for (i64 idx = P.block_colptr(r2); idx <= P.block_colptr(r2 + 1) - 1; ++idx) {
        i64 r1 = P.block_rowval(idx);
        for (i64 r_row = 1; r_row <= st.r_dims(r1); ++r_row) P.S_rowval.push(st.boffsets_r(r1) + r_row - 1);
      }
    }
  }
  P.diag_inds = IV(st.nr);                                                // find_diag_inds (src/utils.jl:82-98)
  for (i64 col = 1; col <= st.nr; ++col) {
    bool found = false;
    for (i64 idx = P.S_colptr(col); idx <= P.S_colptr(col + 1) - 1; ++idx)
      if (P.S_rowval(idx) == col) { P.diag_inds(col) = idx; found = true; break; }
    if (!found) arg_error("column " + std::to_string(col) + " has no stored diagonal entry");
  }
  return P;
}

// The retained part R of a sparse SchurBlockHessian: SparseBlockLinearSystem{T}(TransposedPattern(block_pattern), r_dims)
// (src/schur_hessian.jl:286, src/SparseBlockLinearSystem.jl:43-64). indicestransposed has the block pattern's colptr and
// rowval; its nzval is each block's data start, assigned row block by row block (lower-triangle blocks, each
// d_row x d_col column-major).
struct RLayout {
  IV it_colptr, it_rowval, it_nzval;   // indicestransposed (columns = R row blocks, rows = R column blocks)
  i64 length = 0;
};
RLayout r_layout(const Structure& st, const Pattern& P) {
  RLayout L;
  L.it_colptr = P.block_colptr;
  L.it_rowval = P.block_rowval;
  L.it_nzval = IV(P.block_rowval.len());
  i64 start = 1, ind = 1;
  for (i64 row = 1; row <= st.nrblocks; ++row) {
    i64 rowwidth = st.r_dims(row);
    for (i64 k = L.it_colptr(row); k <= L.it_colptr(row + 1) - 1; ++k) {
      i64 col = L.it_rowval(k);
      L.it_nzval(ind) = start;
      ind += 1;
      start += rowwidth * st.r_dims(col);
    }
  }
  L.length = start - 1;
  return L;
}

// build_r_to_s_map, block-level form (src/schur_structure.jl:406-431). 0 marks an unmapped entry.
IV build_r_to_s_map(const Structure& st, const Pattern& P, const RLayout& L) {
  IV r_to_s(L.length, 0);
  // findnz(indicestransposed): (row = bcol, col = brow, data_start) in CSC order
  for (i64 brow = 1; brow <= st.nrblocks; ++brow) {
    for (i64 k = L.it_colptr(brow); k <= L.it_colptr(brow + 1) - 1; ++k) {
      i64 bcol = L.it_rowval(k), data_start = L.it_nzval(k);
      if (!(brow >= bcol)) continue;
      i64 drow = st.r_dims(brow), dcol = st.r_dims(bcol);
      i64 lo = P.block_colptr(brow), hi = P.block_colptr(brow + 1) - 1;
      i64 idx = lo;
      while (idx <= hi && P.block_rowval(idx) < bcol) ++idx;   // searchsortedfirst
      if (!(idx <= hi && P.block_rowval(idx) == bcol)) throw BlsError(ORC_EPATTERN, "Block of R is not present in the pattern of S");
      i64 row_offset = P.block_row_offsets(idx);
      i64 base = P.S_colptr(st.boffsets_r(brow)) + row_offset;
      i64 stride = P.col_heights(brow);
      if (brow == bcol) {
        for (i64 col = 1; col <= dcol; ++col)
          for (i64 row = 1; row <= col; ++row) r_to_s(data_start + (col - 1) * drow + row - 1) = base + (col - 1) * stride + row - 1;
      } else {
        for (i64 col = 1; col <= dcol; ++col)
          for (i64 row = 1; row <= drow; ++row) r_to_s(data_start + (col - 1) * drow + row - 1) = base + (row - 1) * stride + col - 1;
      }
    }
  }
  return r_to_s;
}

// ------------------------------------------------------------------------------------------------------------------
// SchurReductionWorkspace (src/schur_reduction.jl:16-92) and partition_columns (:30-49)
// ------------------------------------------------------------------------------------------------------------------
std::vector<Range> partition_columns(const IV& retained_ptr, i64 K) {
  i64 n = retained_ptr.len() - 1;
  i64 total = retained_ptr(n + 1) - retained_ptr(1) + n;
  std::vector<Range> ranges;
  i64 start = 1;
  for (i64 k = 1; k <= K; ++k) {
    i64 stop = start - 1;
    if (k == K) stop = n;
    else {
      double target = (double)(total * k) / (double)K;
      while (stop < n && (double)(retained_ptr(stop + 2) - retained_ptr(1) + (stop + 1)) <= target) stop += 1;
    }
    ranges.push_back({start, stop});
    start = stop + 1;
  }
  return ranges;
}

template <class T>
struct Work {
  std::vector<T> W_data, E_inv_data;
  std::vector<double> z_data;
  IV retained_ptr, retained_entry, entry_eliminated;
  std::vector<Range> col_chunks;
  std::atomic<i64> failed_block{0};
};

template <class T>
Work<T>* make_work(const Structure& st, i64 nchunks) {
  auto* ws = new Work<T>();
  i64 total_r = 0, total_e = 0;
  for (i64 d : st.e_dims.v) { total_r += d * d; total_e += d; }
  ws->E_inv_data.assign((size_t)total_r, T(0));
  ws->z_data.assign((size_t)total_e, 0.0);
  i64 ncoup = st.entry_retained.len();
  i64 total_c = 0;
  for (i64 e = 1; e <= st.neblocks; ++e)
    for (i64 c = st.eliminated_ptr(e); c <= st.eliminated_ptr(e + 1) - 1; ++c) total_c += st.r_dims(st.entry_retained(c)) * st.e_dims(e);
  ws->W_data.assign((size_t)total_c, T(0));
  ws->entry_eliminated = IV(ncoup);
  IV counts(st.nrblocks + 1, 0);
  for (i64 e = 1; e <= st.neblocks; ++e)
    for (i64 c = st.eliminated_ptr(e); c <= st.eliminated_ptr(e + 1) - 1; ++c) {
      ws->entry_eliminated(c) = e;
      counts(st.entry_retained(c) + 1) += 1;
    }
  ws->retained_ptr = IV(st.nrblocks + 1);   // cumsum(vcat(1, counts[2:end]))
  ws->retained_ptr(1) = 1;
  for (i64 r = 1; r <= st.nrblocks; ++r) ws->retained_ptr(r + 1) = ws->retained_ptr(r) + counts(r + 1);
  ws->retained_entry = IV(ncoup);
  IV fill_pos = ws->retained_ptr;
  for (i64 c = 1; c <= ncoup; ++c) {
    i64 r = st.entry_retained(c);
    ws->retained_entry(fill_pos(r)) = c;
    fill_pos(r) += 1;
  }
  ws->col_chunks = partition_columns(ws->retained_ptr, std::max<i64>(nchunks, 1));
  return ws;
}

// ------------------------------------------------------------------------------------------------------------------
// Kernels (src/kernels.jl) and conditioning helpers (src/conditioning.jl)
// ------------------------------------------------------------------------------------------------------------------
template <class T> constexpr T eps_of() { return std::numeric_limits<T>::epsilon(); }
template <class T> T singular_tol() { return T(4504) * eps_of<T>(); }   // src/kernels.jl:3

template <class T> inline T scaled(double a, double f) { return T(a * f); }   // src/conditioning.jl:99

inline bool jfinite(double x) { return std::isfinite(x); }

// inv_sym_block closed forms (src/kernels.jl:14-67). Hd is the damped diagonal added as lambda*scale, lambda = 1.
template <class T>
bool inv_sym_1(const T* H, const T* damp, T* inv) {
  T h11 = H[0] + T(1) * damp[0];
  if (!(h11 > T(0)) || !jfinite((double)h11)) { inv[0] = T(0); return false; }
  inv[0] = T(1) / h11;
  return true;
}
template <class T>
bool inv_sym_2(const T* H, const T* damp, T* inv) {   // H column-major 2x2
  T H11 = H[0] + T(1) * damp[0], H22 = H[3] + T(1) * damp[1], H12 = H[2];
  T det = H11 * H22 - H12 * H12;
  if (!(H11 > T(0)) || !(det > singular_tol<T>() * (H11 * H22)) || !jfinite((double)det)) { for (int i = 0; i < 4; ++i) inv[i] = T(0); return false; }
  T inv_det = T(1) / det;
  inv[0] = H22 * inv_det; inv[1] = -H12 * inv_det; inv[2] = -H12 * inv_det; inv[3] = H11 * inv_det;
  return true;
}
template <class T>
bool inv_sym_3(const T* H, const T* damp, T* inv) {   // H column-major 3x3: H[i + 3j]
  T H11 = H[0] + T(1) * damp[0], H22 = H[4] + T(1) * damp[1], H33 = H[8] + T(1) * damp[2];
  T H12 = H[3], H13 = H[6], H23 = H[7];   // H[1,2], H[1,3], H[2,3] (upper triangle)
  T c11 = H22 * H33 - H23 * H23;
  T c12 = H13 * H23 - H12 * H33;
  T c13 = H12 * H23 - H13 * H22;
  T c22 = H11 * H33 - H13 * H13;
  T c23 = H12 * H13 - H11 * H23;
  T c33 = H11 * H22 - H12 * H12;
  T det = H11 * c11 + H12 * c12 + H13 * c13;
  if (!(H11 > T(0)) || !(c33 > singular_tol<T>() * (H11 * H22)) || !(det > singular_tol<T>() * (c33 * H33)) || !jfinite((double)det)) {
    for (int i = 0; i < 9; ++i) inv[i] = T(0);
    return false;
  }
  T inv_det = T(1) / det;
  T v[9] = {c11 * inv_det, c12 * inv_det, c13 * inv_det, c12 * inv_det, c22 * inv_det, c23 * inv_det, c13 * inv_det, c23 * inv_det, c33 * inv_det};
  for (int i = 0; i < 9; ++i) inv[i] = v[i];
  return true;
}
// Generic path (src/kernels.jl:69-83 for d <= 8; src/schur_reduction.jl:173-197 for d > 8), restated from the
// mathematics: upper Cholesky U of the damped block, every pivot^2 / damped diagonal > singular_tol, inverse U^-1 U^-T.
// The reference calls StaticArrays / LAPACK here, so this path is pinned by tolerance, not bit for bit.
template <class T>
bool inv_sym_generic(const T* H, const T* damp, T* inv, int d, const double* hdiag64) {
  std::vector<T> U((size_t)d * d, T(0));
  for (int j = 0; j < d; ++j)
    for (int i = 0; i <= j; ++i) U[i + d * j] = H[i + d * j] + (i == j ? T(1) * damp[i] : T(0));
  std::vector<T> Hd = U;
  for (int j = 0; j < d; ++j) {
    T s = U[j + d * j];
    for (int k = 0; k < j; ++k) s -= U[k + d * j] * U[k + d * j];
    if (!(s > T(0)) || !jfinite((double)s)) { std::fill(inv, inv + d * d, T(0)); return false; }
    T ujj = std::sqrt(s);
    U[j + d * j] = ujj;
    for (int i = j + 1; i < d; ++i) {
      T t = U[j + d * i];
      for (int k = 0; k < j; ++k) t -= U[k + d * j] * U[k + d * i];
      U[j + d * i] = t / ujj;
    }
  }
  for (int i = 0; i < d; ++i) {
    double hii = hdiag64 ? hdiag64[i] : (double)Hd[i + d * i];
    double ratio = ((double)U[i + d * i] * (double)U[i + d * i]) / hii;
    if (!(std::isfinite(ratio) && ratio > (double)singular_tol<T>())) { std::fill(inv, inv + d * d, T(0)); return false; }
  }
  // Uinv (upper), then inv = Uinv * Uinv^T
  std::vector<T> Ui((size_t)d * d, T(0));
  for (int j = 0; j < d; ++j) {
    Ui[j + d * j] = T(1) / U[j + d * j];
    for (int i = j - 1; i >= 0; --i) {
      T s = T(0);
      for (int k = i + 1; k <= j; ++k) s += U[i + d * k] * Ui[k + d * j];
      Ui[i + d * j] = -s / U[i + d * i];
    }
  }
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      T s = T(0);
      for (int k = std::max(i, j); k < d; ++k) s += Ui[i + d * k] * Ui[j + d * k];
      inv[i + d * j] = s;
    }
  return true;
}

// factor_eliminated! (src/schur_reduction.jl:121-162; the d > 8 form :164-225 shares the arithmetic of the inverse's
// consumers). s_r / s_e null means UnitScale (entries 1.0).
template <class T>
bool factor_eliminated(Work<T>& ws, const Structure& st, const T* E_data, const T* C_data, const double* b_e,
                       const double* scaling_e, double lambda, i64 e, const double* s_r, const double* s_e) {
  i64 de = st.e_dims(e);
  i64 eo = st.eoffsets(e), sc_off = st.boffsets_e(e);
  auto SE = [&](i64 i) { return s_e ? s_e[i - 1] : 1.0; };
  auto SR = [&](i64 i) { return s_r ? s_r[i - 1] : 1.0; };
  std::vector<double> se((size_t)de);
  for (i64 i = 1; i <= de; ++i) se[i - 1] = SE(sc_off + i - 1);
  std::vector<T> damp((size_t)de), Es((size_t)(de * de)), Einv((size_t)(de * de));
  for (i64 i = 1; i <= de; ++i) damp[i - 1] = T((lambda * scaling_e[sc_off + i - 2]) * (se[i - 1] * se[i - 1]));
  for (i64 k = 1; k <= de * de; ++k) {
    i64 i = (k - 1) % de + 1, j = (k - 1) / de + 1;
    Es[k - 1] = scaled<T>((double)E_data[eo + k - 2], se[i - 1] * se[j - 1]);
  }
  bool ok;
  if (de == 1) ok = inv_sym_1<T>(Es.data(), damp.data(), Einv.data());
  else if (de == 2) ok = inv_sym_2<T>(Es.data(), damp.data(), Einv.data());
  else if (de == 3) ok = inv_sym_3<T>(Es.data(), damp.data(), Einv.data());
  else if (de <= 8) ok = inv_sym_generic<T>(Es.data(), damp.data(), Einv.data(), (int)de, nullptr);
  else {
    // d > 8 (src/schur_reduction.jl:173-190): M formed with the damping in Float64; pivots judged against the damped
    // diagonal recomputed in Float64 from the inputs
    std::vector<double> hii((size_t)de);
    std::vector<T> dampT((size_t)de);
    for (i64 i = 1; i <= de; ++i) {
      double si = se[i - 1];
      T mii = T((double)Es[(i - 1) * (de + 1)] + lambda * scaling_e[sc_off + i - 2] * (si * si));
      dampT[i - 1] = mii - Es[(i - 1) * (de + 1)];
      hii[i - 1] = (double)E_data[eo + (i - 1) * (de + 1) - 1] * (si * si) + lambda * scaling_e[sc_off + i - 2] * (si * si);
    }
    ok = inv_sym_generic<T>(Es.data(), dampT.data(), Einv.data(), (int)de, hii.data());
  }
  if (!ok) return false;
  for (i64 i = 1; i <= de * de; ++i) ws.E_inv_data[eo + i - 2] = Einv[i - 1];
  // z_e = E_inv * (b_e .* se): promoted to Float64 (src/schur_reduction.jl:144-147)
  for (i64 i = 1; i <= de; ++i) {
    double acc = (double)Einv[(i - 1)] * (b_e[sc_off - 1] * se[0]);
    for (i64 j = 2; j <= de; ++j) acc = acc + (double)Einv[(i - 1) + (j - 1) * de] * (b_e[sc_off + j - 2] * se[j - 1]);
    ws.z_data[sc_off + i - 2] = acc;
  }
  // W_er = E_inv * scaled C column (src/schur_reduction.jl:149-160), in T
  std::vector<T> cs((size_t)de);
  for (i64 c = st.eliminated_ptr(e); c <= st.eliminated_ptr(e + 1) - 1; ++c) {
    i64 co = st.coffsets(c), r = st.entry_retained(c), dr = st.r_dims(r), ro = st.boffsets_r(r);
    for (i64 ir = 1; ir <= dr; ++ir) {
      double f = SR(ro + ir - 1);
      for (i64 i = 1; i <= de; ++i) cs[i - 1] = scaled<T>((double)C_data[co + (ir - 1) * de + i - 2], SE(sc_off + i - 1) * f);
      for (i64 i = 1; i <= de; ++i) {
        T acc = Einv[i - 1] * cs[0];
        for (i64 j = 2; j <= de; ++j) acc = acc + Einv[(i - 1) + (j - 1) * de] * cs[j - 1];
        ws.W_data[co + (ir - 1) * de + i - 2] = acc;
      }
    }
  }
  return true;
}

inline bool use_threads(i64 nitems, i64 work, i64 min_work, int nthreads) { return nitems > 1 && work >= min_work && nthreads > 1; }

// factor_eliminated_group! (src/schur_reduction.jl:233-257) + factor_all_eliminated! (:439-455)
template <class T>
bool factor_all(Work<T>& ws, const Structure& st, const T* E, const T* C, const double* b_e, const double* sc_e,
                double lambda, const double* s_r, const double* s_e, int nthreads) {
  for (i64 g = 1; g <= st.e_runs.nruns(); ++g) {
    const auto& chunks = st.chunks[g - 1];
    bool threaded = use_threads((i64)chunks.size(), st.entry_retained.len(), st.min_work, nthreads);
    i64 nk = (i64)chunks.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (threaded)
    for (i64 k = 1; k <= nk; ++k) {
      for (i64 e = chunks[k - 1].first; e <= chunks[k - 1].last; ++e) {
        i64 fb = ws.failed_block.load();
        if (fb != 0 && e > fb) break;
        if (!factor_eliminated<T>(ws, st, E, C, b_e, sc_e, lambda, e, s_r, s_e)) {
          i64 old = ws.failed_block.load();
          while (old == 0 || e < old) {
            if (ws.failed_block.compare_exchange_weak(old, e)) break;
          }
          break;
        }
      }
    }
    if (ws.failed_block.load() != 0) return false;
  }
  return true;
}

// check_damping (src/utils.jl:100-107)
void check_damping(double lambda, const double* scaling, i64 n, const char* name) {
  if (!(std::isfinite(lambda) && lambda >= 0)) arg_error("lambda must be finite and non-negative");
  for (i64 i = 0; i < n; ++i)
    if (!(std::isfinite(scaling[i]) && scaling[i] >= 0)) arg_error(std::string(name) + " must be finite and non-negative");
}

// accumulate_entry_sparse! (src/schur_reduction.jl:315-354) over accumulate_sparse_columns! (:362-387)
template <class T>
void accumulate_sparse_columns(T* nzval, double* g_S, const Structure& st, const T* C_data, const Work<T>& ws,
                               const Pattern& P, Range r_range, const double* s_r, const double* s_e) {
  auto SE = [&](i64 i) { return s_e ? s_e[i - 1] : 1.0; };
  auto SR = [&](i64 i) { return s_r ? s_r[i - 1] : 1.0; };
  std::vector<T> cs(64);
  for (i64 r2 = r_range.first; r2 <= r_range.last; ++r2) {
    for (i64 kk = ws.retained_ptr(r2); kk <= ws.retained_ptr(r2 + 1) - 1; ++kk) {
      i64 c2 = ws.retained_entry(kk), e = ws.entry_eliminated(c2);
      i64 de = st.e_dims(e);
      if ((i64)cs.size() < de) cs.resize((size_t)de);
      i64 dr2 = st.r_dims(r2), ro2 = st.boffsets_r(r2), co2 = st.coffsets(c2), sc_off = st.boffsets_e(e);
      for (i64 ir = 1; ir <= dr2; ++ir) {
        double f = SR(ro2 + ir - 1);
        double acc = 0.0;   // dot_col(v, b, ib): promote(T, Float64) = Float64, from zero
        for (i64 i = 0; i <= de - 1; ++i)
          acc = acc + (double)scaled<T>((double)C_data[co2 + (ir - 1) * de + i - 1], SE(sc_off + i) * f) * ws.z_data[sc_off + i - 1];
        g_S[ro2 + ir - 2] -= acc;
      }
      i64 col_base = P.S_colptr(ro2), stride = P.col_heights(r2);
      i64 b_row_idx = P.block_colptr(r2), b_row_end = P.block_colptr(r2 + 1) - 1;
      for (i64 c1 = st.eliminated_ptr(e); c1 <= c2; ++c1) {
        i64 r1 = st.entry_retained(c1), dr1 = st.r_dims(r1), wo1 = st.coffsets(c1);
        while (b_row_idx <= b_row_end && P.block_rowval(b_row_idx) < r1) b_row_idx += 1;
        if (!(b_row_idx <= b_row_end && P.block_rowval(b_row_idx) == r1)) throw BlsError(ORC_EPATTERN, "The sparse pattern has no block");
        i64 row_offset = P.block_row_offsets(b_row_idx);
        for (i64 col = 1; col <= dr2; ++col) {
          i64 c_off = co2 + (col - 1) * de;
          double f = SR(ro2 + col - 1);
          for (i64 i = 1; i <= de; ++i) cs[i - 1] = scaled<T>((double)C_data[c_off + i - 2], SE(sc_off + i - 1) * f);
          i64 col_ptr = col_base + (col - 1) * stride + row_offset;
          i64 nrow = r1 == r2 ? col : dr1;
          for (i64 row = 1; row <= nrow; ++row) {
            T acc = T(0);   // dot_col(a, ia, v): promote(T, T) = T, from zero
            for (i64 i = 0; i <= de - 1; ++i) acc = acc + ws.W_data[wo1 + (row - 1) * de + i - 1] * cs[i];
            nzval[col_ptr + row - 2] -= acc;
          }
        }
      }
    }
  }
}

// accumulate_entry_dense! (src/schur_reduction.jl:262-296) over accumulate_dense_columns! (:298-313). S column-major nr x nr.
template <class T>
void accumulate_dense_columns(T* S, i64 nr, double* g_S, const Structure& st, const T* C_data, const Work<T>& ws,
                              Range r_range, const double* s_r, const double* s_e) {
  auto SE = [&](i64 i) { return s_e ? s_e[i - 1] : 1.0; };
  auto SR = [&](i64 i) { return s_r ? s_r[i - 1] : 1.0; };
  std::vector<T> cs(64);
  for (i64 r2 = r_range.first; r2 <= r_range.last; ++r2) {
    for (i64 kk = ws.retained_ptr(r2); kk <= ws.retained_ptr(r2 + 1) - 1; ++kk) {
      i64 c2 = ws.retained_entry(kk), e = ws.entry_eliminated(c2);
      i64 de = st.e_dims(e);
      if ((i64)cs.size() < de) cs.resize((size_t)de);
      i64 dr2 = st.r_dims(r2), ro2 = st.boffsets_r(r2), co2 = st.coffsets(c2), sc_off = st.boffsets_e(e);
      for (i64 ir = 1; ir <= dr2; ++ir) {
        double f = SR(ro2 + ir - 1);
        double acc = 0.0;
        for (i64 i = 0; i <= de - 1; ++i)
          acc = acc + (double)scaled<T>((double)C_data[co2 + (ir - 1) * de + i - 1], SE(sc_off + i) * f) * ws.z_data[sc_off + i - 1];
        g_S[ro2 + ir - 2] -= acc;
      }
      for (i64 c1 = st.eliminated_ptr(e); c1 <= c2; ++c1) {
        i64 r1 = st.entry_retained(c1), dr1 = st.r_dims(r1), ro1 = st.boffsets_r(r1), wo1 = st.coffsets(c1);
        for (i64 col = 1; col <= dr2; ++col) {
          i64 c_off = co2 + (col - 1) * de;
          double f = SR(ro2 + col - 1);
          for (i64 i = 1; i <= de; ++i) cs[i - 1] = scaled<T>((double)C_data[c_off + i - 2], SE(sc_off + i - 1) * f);
          i64 nrow = r1 == r2 ? col : dr1;
          for (i64 row = 1; row <= nrow; ++row) {
            T acc = T(0);
            for (i64 i = 0; i <= de - 1; ++i) acc = acc + ws.W_data[wo1 + (row - 1) * de + i - 1] * cs[i];
            S[(ro1 + row - 2) + (ro2 + col - 2) * nr] -= acc;
          }
        }
      }
    }
  }
}

// reset_schur_sparse! (src/schur_reduction.jl:416-436) with scale_sparse! (src/conditioning.jl:144-150)
template <class T>
void reset_sparse(T* nzval, i64 nnz, const T* R_nzval, const IV& r_to_s, const IV& diag_inds, const double* scaling_r,
                  i64 nr, double lambda, const double* s_r, const IV* S_colptr, const IV* S_rowval) {
  check_damping(lambda, scaling_r, nr, "scaling_r");
  for (i64 i = 0; i < nnz; ++i) nzval[i] = T(0);
  for (i64 i = 1; i <= r_to_s.len(); ++i) {
    i64 idx = r_to_s(i);
    if (idx > 0) nzval[idx - 1] = R_nzval[i - 1];
  }
  if (s_r) {
    for (i64 j = 1; j <= nr; ++j)
      for (i64 k = (*S_colptr)(j); k <= (*S_colptr)(j + 1) - 1; ++k)
        nzval[k - 1] = scaled<T>((double)nzval[k - 1], s_r[(*S_rowval)(k) - 1] * s_r[j - 1]);
  }
  for (i64 i = 1; i <= diag_inds.len(); ++i) {
    double si = s_r ? s_r[i - 1] : 1.0;
    i64 idx = diag_inds(i);
    nzval[idx - 1] = T((double)nzval[idx - 1] + lambda * scaling_r[i - 1] * (si * si));
  }
}

// reset_schur_dense! (src/schur_reduction.jl:389-407)
template <class T>
void reset_dense(T* S, const T* R, const double* scaling_r, i64 nr, double lambda, const double* s_r) {
  check_damping(lambda, scaling_r, nr, "scaling_r");
  if (!s_r) std::memcpy(S, R, sizeof(T) * (size_t)(nr * nr));
  else
    for (i64 j = 1; j <= nr; ++j)
      for (i64 i = 1; i <= nr; ++i) S[(i - 1) + (j - 1) * nr] = scaled<T>((double)R[(i - 1) + (j - 1) * nr], s_r[i - 1] * s_r[j - 1]);
  for (i64 i = 1; i <= nr; ++i) {
    double si = s_r ? s_r[i - 1] : 1.0;
    S[(i - 1) * (nr + 1)] = T((double)S[(i - 1) * (nr + 1)] + lambda * scaling_r[i - 1] * (si * si));
  }
}

// backsubstitute_group! (src/schur_reduction.jl:541-614) over backsubstitute! (:519-538). x_e, x_r, z, t in Float64.
template <class T>
void backsubstitute(double* x_e, const double* x_r, const Structure& st, const T* C_data, const Work<T>& ws,
                    const double* s_r, const double* s_e, int nthreads) {
  auto SE = [&](i64 i) { return s_e ? s_e[i - 1] : 1.0; };
  auto SR = [&](i64 i) { return s_r ? s_r[i - 1] : 1.0; };
  for (i64 g = 1; g <= st.e_runs.nruns(); ++g) {
    const auto& chunks = st.chunks[g - 1];
    bool threaded = use_threads((i64)chunks.size(), st.entry_retained.len(), st.min_work, nthreads);
    i64 nk = (i64)chunks.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (threaded)
    for (i64 k = 1; k <= nk; ++k) {
      std::vector<double> t(64);
      for (i64 e = chunks[k - 1].first; e <= chunks[k - 1].last; ++e) {
        i64 de = st.e_dims(e), e_off = st.boffsets_e(e), eo = st.eoffsets(e);
        if ((i64)t.size() < de) t.resize((size_t)de);
        for (i64 i = 0; i < de; ++i) t[i] = 0.0;
        for (i64 c = st.eliminated_ptr(e); c <= st.eliminated_ptr(e + 1) - 1; ++c) {
          i64 r = st.entry_retained(c), dr = st.r_dims(r), ro = st.boffsets_r(r), co = st.coffsets(c);
          for (i64 ir = 1; ir <= dr; ++ir) {
            double xc = x_r[ro + ir - 2], f = SR(ro + ir - 1);
            for (i64 i = 1; i <= de; ++i) t[i - 1] = t[i - 1] + (double)scaled<T>((double)C_data[co + (ir - 1) * de + i - 2], SE(e_off + i - 1) * f) * xc;
          }
        }
        for (i64 i = 1; i <= de; ++i) {
          double acc = (double)ws.E_inv_data[eo + (i - 1) - 1] * t[0];
          for (i64 j = 2; j <= de; ++j) acc = acc + (double)ws.E_inv_data[eo + (j - 1) * de + i - 2] * t[j - 1];
          x_e[e_off + i - 2] = ws.z_data[e_off + i - 2] - acc;
        }
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------------------------
// QR elimination: SchurJacobianStructure (src/schur_jacobian.jl:59-160, src/schur_description.jl:137-189)
// ------------------------------------------------------------------------------------------------------------------
struct QRStructure {
  Structure schur;
  IV e_rows, free_rows, table_nrows, table_ncols, table_top, table_offsets, raw_offsets, residual_offsets, table_ptr;
  IV entry_retained, entry_col, entry_table, retained_ptr, retained_entry, reduced_offsets, doffsets;
  std::vector<Range> col_chunks;
  i64 ntables = 0;
  IV row_table, row_first, row_nrows, row_ptr, row_blocks;
};

QRStructure make_qr_structure(const Structure& st, const IV& e_rows, const IV& free_rows, const std::vector<std::vector<i64>>& free_retained, i64 nchunks) {
  QRStructure q;
  q.schur = st;
  i64 ne = st.neblocks, nrb = st.nrblocks, nfree = free_rows.len();
  if (e_rows.len() != ne) dim_error("Number of eliminated row counts must match the number of eliminated blocks");
  if ((i64)free_retained.size() != nfree) dim_error("Number of free groups' retained lists must match the number of free row counts");
  if (nchunks < 1) arg_error("nchunks must be at least 1");
  for (i64 e = 1; e <= ne; ++e) if (e_rows(e) < 1) arg_error("Eliminated block needs at least 1 row");
  for (i64 g = 1; g <= nfree; ++g) if (free_rows(g) < 1) arg_error("Free group needs at least 1 row");
  IV seen(nrb, 0);
  for (i64 g = 1; g <= nfree; ++g)
    for (i64 r : free_retained[g - 1]) {
      if (!(1 <= r && r <= nrb)) arg_error("Free group references a missing retained block");
      if (seen(r) == g) arg_error("Retained block listed more than once in a free group");
      seen(r) = g;
    }
  i64 ntables = ne + nfree;
  q.ntables = ntables;
  std::vector<std::vector<i64>> sorted_free = free_retained;
  for (auto& s : sorted_free) std::sort(s.begin(), s.end());
  q.table_nrows = IV(ntables); q.table_ncols = IV(ntables); q.table_top = IV(ntables); q.table_ptr = IV(ntables + 1);
  i64 u = 1;
  q.table_ptr(1) = 1;
  for (i64 t = 1; t <= ntables; ++t) {
    std::vector<i64> rs;
    if (t <= ne) for (i64 c = st.eliminated_ptr(t); c <= st.eliminated_ptr(t + 1) - 1; ++c) rs.push_back(st.entry_retained(c));
    else rs = sorted_free[t - ne - 1];
    i64 col = 1;
    for (i64 r : rs) {
      q.entry_retained.push(r); q.entry_col.push(col); q.entry_table.push(t);
      col += st.r_dims(r);
      u += 1;
    }
    q.table_ptr(t + 1) = u;
    i64 de = t <= ne ? st.e_dims(t) : 0;
    q.table_top(t) = de;
    q.table_nrows(t) = t <= ne ? e_rows(t) + de : free_rows(t - ne);
    q.table_ncols(t) = col - 1 + de + 1;
  }
  q.table_offsets = IV(ntables + 1); q.raw_offsets = IV(ntables + 1); q.residual_offsets = IV(ntables + 1); q.reduced_offsets = IV(ntables + 1);
  q.table_offsets(1) = q.raw_offsets(1) = q.residual_offsets(1) = q.reduced_offsets(1) = 1;
  for (i64 t = 1; t <= ntables; ++t) {
    q.table_offsets(t + 1) = q.table_offsets(t) + q.table_nrows(t) * q.table_ncols(t);
    q.raw_offsets(t + 1) = q.raw_offsets(t) + q.table_nrows(t) * (q.table_ncols(t) - 1);
    q.residual_offsets(t + 1) = q.residual_offsets(t) + q.table_nrows(t);
    q.reduced_offsets(t + 1) = q.reduced_offsets(t) + q.table_nrows(t) - q.table_top(t);
  }
  i64 nentries = q.entry_retained.len();
  IV counts(nrb + 1, 0);
  for (i64 uu = 1; uu <= nentries; ++uu) counts(q.entry_retained(uu) + 1) += 1;
  q.retained_ptr = IV(nrb + 1);
  q.retained_ptr(1) = 1;
  for (i64 r = 1; r <= nrb; ++r) q.retained_ptr(r + 1) = q.retained_ptr(r) + counts(r + 1);
  q.retained_entry = IV(nentries);
  IV fill_pos = q.retained_ptr;
  for (i64 uu = 1; uu <= nentries; ++uu) { i64 r = q.entry_retained(uu); q.retained_entry(fill_pos(r)) = uu; fill_pos(r) += 1; }
  q.doffsets = IV(nrb + 1);
  q.doffsets(1) = 1;
  for (i64 r = 1; r <= nrb; ++r) q.doffsets(r + 1) = q.doffsets(r) + st.r_dims(r) * st.r_dims(r);
  q.col_chunks = partition_columns(q.retained_ptr, nchunks);
  return q;
}

// SchurJacobianStructure(blocksizes, rowblocks, rowblocksizes; eliminated) (src/schur_description.jl:137-189)
QRStructure qr_structure_from_description(const IV& blocksizes, const std::vector<std::vector<i64>>& rowblocks, const IV& rowblocksizes,
                                          const std::vector<bool>& eliminated, i64 nchunks, i64 min_work) {
  Structure st = structure_from_description(blocksizes, rowblocks, eliminated, &rowblocksizes, nchunks, min_work);
  i64 nret = st.nrblocks, ne = st.neblocks, K = (i64)rowblocks.size();
  IV row_table(K), row_first(K), e_rows(ne, 0), row_ptr(K + 1), free_rows_v;
  std::map<std::vector<i64>, i64> group;
  std::vector<std::vector<i64>> free_retained;
  row_ptr(1) = 1;
  for (i64 k = 1; k <= K; ++k) row_ptr(k + 1) = row_ptr(k) + (i64)rowblocks[k - 1].size();
  IV row_blocks(row_ptr(K + 1) - 1);
  for (i64 k = 1; k <= K; ++k) {
    i64 m = rowblocksizes(k), i = row_ptr(k);
    for (i64 b : rowblocks[k - 1]) { row_blocks(i) = st.position(b); i += 1; }
    std::sort(row_blocks.v.begin() + (row_ptr(k) - 1), row_blocks.v.begin() + (row_ptr(k + 1) - 1));
    i64 e = st.rowblock_eliminated(k);
    if (e != 0) {
      i64 t = st.position(e) - nret;
      row_table(k) = t;
      row_first(k) = e_rows(t) + 1;
      e_rows(t) += m;
    } else {
      std::vector<i64> rs(row_blocks.v.begin() + (row_ptr(k) - 1), row_blocks.v.begin() + (row_ptr(k + 1) - 1));
      auto it = group.find(rs);
      i64 g;
      if (it == group.end()) {
        free_retained.push_back(rs);
        free_rows_v.push(0);
        g = free_rows_v.len();
        group[rs] = g;
      } else g = it->second;
      row_table(k) = ne + g;
      row_first(k) = free_rows_v(g) + 1;
      free_rows_v(g) += m;
    }
  }
  QRStructure q = make_qr_structure(st, e_rows, free_rows_v, free_retained, nchunks);
  q.e_rows = e_rows; q.free_rows = free_rows_v;
  q.row_table = row_table; q.row_first = row_first; q.row_nrows = rowblocksizes; q.row_ptr = row_ptr; q.row_blocks = row_blocks;
  return q;
}

// copy_table! (src/qr_reduction.jl:192-221) + scale_table_columns! (:225-255); s null = UnitScale
template <class T>
bool copy_table(T* F, double* Fr, const T* Rw, const double* Rr, const QRStructure& q, i64 t, const double* s) {
  i64 M = q.table_nrows(t), C = q.table_ncols(t) - 1, off = q.raw_offsets(t);
  T bad = T(0);
  if (!s) {
    for (i64 i = off; i <= off + M * C - 1; ++i) { T x = Rw[i - 1]; F[i - 1] = x; bad += x - x; }
  } else {
    for (i64 i = off; i <= off + M * C - 1; ++i) { T x = Rw[i - 1]; bad += x - x; }
    const Structure& st = q.schur;
    for (i64 u = q.table_ptr(t); u <= q.table_ptr(t + 1) - 1; ++u) {
      i64 r = q.entry_retained(u), ro = st.boffsets_r(r);
      for (i64 k = 1; k <= st.r_dims(r); ++k) {
        double f = s[ro + k - 2];
        i64 cb = off + (q.entry_col(u) + k - 2) * M;
        for (i64 i = cb; i <= cb + M - 1; ++i) F[i - 1] = scaled<T>((double)Rw[i - 1], f);
      }
    }
    if (t <= st.neblocks) {
      i64 de = st.e_dims(t), eo = st.nr + st.boffsets_e(t) - 1;
      for (i64 k = 1; k <= de; ++k) {
        double f = s[eo + k - 1];
        i64 cb = off + (C - de + k - 1) * M;
        for (i64 i = cb; i <= cb + M - 1; ++i) F[i - 1] = scaled<T>((double)Rw[i - 1], f);
      }
    }
  }
  i64 rb = q.residual_offsets(t);
  double badr = 0.0;
  for (i64 i = rb; i <= rb + M - 1; ++i) { double x = Rr[i - 1]; Fr[i - 1] = x; badr += x - x; }
  return !std::isnan((double)bad) && !std::isnan(badr);
}

// qr_table! (src/qr_reduction.jl:50-131)
template <class T>
bool qr_table(T* F, double* Fr, const T* Rw, const double* Rr, const QRStructure& q, const double* scaling_e, double lambda, i64 e, const double* cs) {
  const Structure& st = q.schur;
  i64 de = st.e_dims(e);
  i64 M = q.table_nrows(e), C = q.table_ncols(e) - 1, off = q.raw_offsets(e), rq = q.residual_offsets(e) - 1;
  i64 me = M - de, ce = C - de;
  if (!copy_table<T>(F, Fr, Rw, Rr, q, e, cs)) return false;
  for (i64 j = 1; j <= C; ++j) for (i64 i = me + 1; i <= M; ++i) F[off + (j - 1) * M + i - 2] = T(0);
  for (i64 i = me + 1; i <= M; ++i) Fr[rq + i - 1] = 0.0;
  i64 so = st.boffsets_e(e), nr = st.nr;
  for (i64 k = 1; k <= de; ++k) {
    double csv = cs ? cs[nr + so + k - 2] : 1.0;
    F[off + (ce + k - 1) * M + me + k - 2] = T(std::sqrt(lambda * scaling_e[so + k - 2]) * csv);
  }
  T tol = T(M) * eps_of<T>();
  for (i64 k = 1; k <= de; ++k) {
    i64 cb = off + (ce + k - 1) * M - 1;   // F[cb + i] is row i (1-based F index)
    auto Fat = [&](i64 idx) -> T& { return F[idx - 1]; };
    T s_top = T(0);
    for (i64 i = 1; i <= k - 1; ++i) s_top += Fat(cb + i) * Fat(cb + i);
    T s_sub = T(0);
    for (i64 i = k; i <= M; ++i) s_sub += Fat(cb + i) * Fat(cb + i);
    T nrm = std::sqrt(s_sub);
    T full = std::sqrt(s_top + s_sub);
    T a = Fat(cb + k);
    T beta = a >= T(0) ? -nrm : nrm;
    if (!(std::isfinite((double)beta) && std::abs(beta) > tol * full)) return false;
    T scale = T(1) / (a - beta);
    for (i64 i = k + 1; i <= M; ++i) Fat(cb + i) *= scale;
    T tau = (beta - a) / beta;
    Fat(cb + k) = beta;
    for (i64 j = 1; j <= C; ++j) {
      if (ce + 1 <= j && j <= ce + k) continue;
      i64 yb = off + (j - 1) * M - 1;
      T s = Fat(yb + k);
      for (i64 i = k + 1; i <= M; ++i) s += Fat(cb + i) * Fat(yb + i);
      s *= tau;
      Fat(yb + k) -= s;
      for (i64 i = k + 1; i <= M; ++i) Fat(yb + i) -= s * Fat(cb + i);
    }
    double sr = Fr[rq + k - 1];
    for (i64 i = k + 1; i <= M; ++i) sr += (double)Fat(cb + i) * Fr[rq + i - 1];
    sr *= (double)tau;
    Fr[rq + k - 1] -= sr;
    for (i64 i = k + 1; i <= M; ++i) Fr[rq + i - 1] -= sr * (double)Fat(cb + i);
    for (i64 i = k + 1; i <= M; ++i) Fat(cb + i) = T(0);
  }
  return true;
}

// reduce_qr! (src/qr_reduction.jl:162-187) with qr_group! (:145-158)
template <class T>
bool reduce_qr(const QRStructure& q, T* F, double* Fr, const T* Rw, const double* Rr, const double* scaling_e, i64 n_sc, double lambda,
               const double* s, int nthreads, i64* failed_out) {
  const Structure& st = q.schur;
  i64 ne_sc = 0; for (i64 d : st.e_dims.v) ne_sc += d;
  if (n_sc != ne_sc) dim_error("scaling_e has the wrong length");
  check_damping(lambda, scaling_e, n_sc, "scaling_e");
  std::atomic<i64> failed{0};
  i64 table_len = q.table_offsets(q.ntables + 1) - 1;
  for (i64 g = 1; g <= st.e_runs.nruns(); ++g) {
    const auto& chunks = st.chunks[g - 1];
    bool threaded = use_threads((i64)chunks.size(), table_len, st.min_work, nthreads);
    i64 nk = (i64)chunks.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (threaded)
    for (i64 k = 1; k <= nk; ++k) {
      for (i64 e = chunks[k - 1].first; e <= chunks[k - 1].last; ++e) {
        i64 fb = failed.load();
        if (fb != 0 && e > fb) break;
        if (!qr_table<T>(F, Fr, Rw, Rr, q, scaling_e, lambda, e, s)) {
          i64 old = failed.load();
          while (old == 0 || e < old) if (failed.compare_exchange_weak(old, e)) break;
          break;
        }
      }
    }
    if (failed.load() != 0) { *failed_out = failed.load(); return false; }
  }
  for (i64 t = st.neblocks + 1; t <= q.ntables; ++t) copy_table<T>(F, Fr, Rw, Rr, q, t, s);
  *failed_out = 0;
  return true;
}

// qr_backsubstitute_group! (src/qr_reduced.jl:24-93): x_e = U^-1 (q - B x_r), in Float64
template <class T>
void qr_backsubstitute(double* x_e, const double* x_r, const T* F, const double* Fr, const QRStructure& q) {
  const Structure& st = q.schur;
  for (i64 e = 1; e <= st.neblocks; ++e) {
    i64 M = q.table_nrows(e), C = q.table_ncols(e), off = q.raw_offsets(e), de = st.e_dims(e), ce = C - de - 1;
    std::vector<double> t((size_t)de);
    for (i64 i = 1; i <= de; ++i) t[i - 1] = Fr[q.residual_offsets(e) + i - 2];
    for (i64 u = q.table_ptr(e); u <= q.table_ptr(e + 1) - 1; ++u) {
      i64 r = q.entry_retained(u), ro = st.boffsets_r(r), cb = off + (q.entry_col(u) - 1) * M;
      for (i64 j = 1; j <= st.r_dims(r); ++j) {
        double xj = x_r[ro + j - 2];
        for (i64 i = 1; i <= de; ++i) t[i - 1] = t[i - 1] - (double)F[cb + (j - 1) * M + i - 2] * xj;
      }
    }
    i64 eo = st.boffsets_e(e);
    for (i64 i = de; i >= 1; --i) {
      double acc = t[i - 1];
      for (i64 j = i + 1; j <= de; ++j) acc -= (double)F[off + (ce + j - 1) * M + i - 2] * x_e[eo + j - 2];
      x_e[eo + i - 2] = acc / (double)F[off + (ce + i - 1) * M + i - 2];
    }
  }
}

// accumulate_qr_entry! (src/qr_reduced.jl:375-405) driven by reduced_normal_sparse! (:440-480)
// Threaded over block columns r2 as foreach_retained threads over column chunks (:116-124): each writes its own columns.
template <class T>
void reduced_normal_sparse(T* nzval, double* g_S, const T* F, const double* Fr, const QRStructure& q, const Pattern& P) {
  const Structure& st = q.schur;
  int missing = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(| : missing)
  for (i64 r2 = 1; r2 <= st.nrblocks; ++r2) {
    i64 ro2 = st.boffsets_r(r2), dr2 = st.r_dims(r2);
    for (i64 i = P.S_colptr(ro2); i <= P.S_colptr(ro2 + dr2) - 1; ++i) nzval[i - 1] = T(0);
    for (i64 col = ro2; col <= ro2 + dr2 - 1; ++col) g_S[col - 1] = 0.0;
    i64 col_base = P.S_colptr(ro2), stride = P.col_heights(r2);
    i64 b_lo = P.block_colptr(r2), b_hi = P.block_colptr(r2 + 1) - 1;
    for (i64 kk = q.retained_ptr(r2); kk <= q.retained_ptr(r2 + 1) - 1; ++kk) {
      i64 u2 = q.retained_entry(kk), t = q.entry_table(u2), M = q.table_nrows(t), top = q.table_top(t), n = M - top;
      i64 off = q.raw_offsets(t) + top, cb2 = off + (q.entry_col(u2) - 1) * M, rb = q.residual_offsets(t) + top;
      for (i64 j = 1; j <= dr2; ++j) {
        double acc = 0.0;
        for (i64 i = 0; i <= n - 1; ++i) acc += (double)F[cb2 + (j - 1) * M + i - 1] * Fr[rb + i - 1];
        g_S[ro2 + j - 2] += acc;
      }
      for (i64 u1 = q.table_ptr(t); u1 <= u2; ++u1) {
        i64 r1 = q.entry_retained(u1), dr1 = st.r_dims(r1), cb1 = off + (q.entry_col(u1) - 1) * M;
        i64 idx = b_lo;
        while (idx <= b_hi && P.block_rowval(idx) < r1) ++idx;
        if (!(idx <= b_hi && P.block_rowval(idx) == r1)) { missing = 1; continue; }
        i64 row_offset = P.block_row_offsets(idx);
        for (i64 col = 1; col <= dr2; ++col) {
          i64 nrow = u1 == u2 ? col : dr1;
          for (i64 row = 1; row <= nrow; ++row) {
            T acc = T(0);
            for (i64 i = 0; i <= n - 1; ++i) acc += F[cb1 + (row - 1) * M + i - 1] * F[cb2 + (col - 1) * M + i - 1];
            nzval[col_base + (col - 1) * stride + row_offset + row - 2] += acc;
          }
        }
      }
    }
  }
  if (missing) throw BlsError(ORC_EPATTERN, "The sparse pattern has no block");
}

// reduced_normal_dense! (src/qr_reduced.jl:409-436)
template <class T>
void reduced_normal_dense(T* S, double* g_S, const T* F, const double* Fr, const QRStructure& q) {
  const Structure& st = q.schur;
  i64 nr = st.nr;
  for (i64 r2 = 1; r2 <= st.nrblocks; ++r2) {
    i64 ro2 = st.boffsets_r(r2), dr2 = st.r_dims(r2);
    for (i64 col = ro2; col <= ro2 + dr2 - 1; ++col) {
      for (i64 row = 1; row <= nr; ++row) S[(row - 1) + (col - 1) * nr] = T(0);
      g_S[col - 1] = 0.0;
    }
    for (i64 kk = q.retained_ptr(r2); kk <= q.retained_ptr(r2 + 1) - 1; ++kk) {
      i64 u2 = q.retained_entry(kk), t = q.entry_table(u2), M = q.table_nrows(t), top = q.table_top(t), n = M - top;
      i64 off = q.raw_offsets(t) + top, cb2 = off + (q.entry_col(u2) - 1) * M, rb = q.residual_offsets(t) + top;
      for (i64 j = 1; j <= dr2; ++j) {
        double acc = 0.0;
        for (i64 i = 0; i <= n - 1; ++i) acc += (double)F[cb2 + (j - 1) * M + i - 1] * Fr[rb + i - 1];
        g_S[ro2 + j - 2] += acc;
      }
      for (i64 u1 = q.table_ptr(t); u1 <= u2; ++u1) {
        i64 r1 = q.entry_retained(u1), dr1 = st.r_dims(r1), ro1 = st.boffsets_r(r1), cb1 = off + (q.entry_col(u1) - 1) * M;
        for (i64 col = 1; col <= dr2; ++col) {
          i64 nrow = u1 == u2 ? col : dr1;
          for (i64 row = 1; row <= nrow; ++row) {
            T acc = T(0);
            for (i64 i = 0; i <= n - 1; ++i) acc += F[cb1 + (row - 1) * M + i - 1] * F[cb2 + (col - 1) * M + i - 1];
            S[(ro1 + row - 2) + (ro2 + col - 2) * nr] += acc;
          }
        }
      }
    }
  }
}

// reduced_diagonal_blocks! (src/qr_reduced.jl:484-512)
template <class T>
void reduced_diagonal_blocks(T* D, const T* F, const QRStructure& q) {
  const Structure& st = q.schur;
  for (i64 r = 1; r <= st.nrblocks; ++r) {
    i64 dr = st.r_dims(r), d0 = q.doffsets(r);
    for (i64 i = d0; i <= d0 + dr * dr - 1; ++i) D[i - 1] = T(0);
    for (i64 kk = q.retained_ptr(r); kk <= q.retained_ptr(r + 1) - 1; ++kk) {
      i64 u = q.retained_entry(kk), t = q.entry_table(u), M = q.table_nrows(t), top = q.table_top(t);
      i64 cb = q.raw_offsets(t) + top + (q.entry_col(u) - 1) * M;
      for (i64 col = 1; col <= dr; ++col)
        for (i64 row = 1; row <= col; ++row) {
          T acc = T(0);
          for (i64 i = 0; i <= M - top - 1; ++i) acc += F[cb + (row - 1) * M + i - 1] * F[cb + (col - 1) * M + i - 1];
          D[d0 + (col - 1) * dr + row - 2] += acc;
        }
    }
    for (i64 col = 1; col <= dr; ++col)
      for (i64 row = col + 1; row <= dr; ++row) D[d0 + (col - 1) * dr + row - 2] = D[d0 + (row - 1) * dr + col - 2];
  }
}

// factor_diagonal_blocks! / solve_diagonal_blocks! (src/diagonal_blocks.jl:6-61)
template <class T>
bool factor_diagonal_blocks(T* D, const i64* dims, i64 nb) {
  i64 o = 0;
  for (i64 b = 0; b < nb; ++b) {
    i64 d = dims[b];
    for (i64 j = 1; j <= d; ++j) {
      T s = D[o + (j - 1) * d + j - 1];
      for (i64 k = 1; k <= j - 1; ++k) { T l = D[o + (k - 1) * d + j - 1]; s -= l * l; }
      if (!(s > T(0) && std::isfinite((double)s))) return false;
      T ljj = std::sqrt(s);
      D[o + (j - 1) * d + j - 1] = ljj;
      for (i64 i = j + 1; i <= d; ++i) {
        T t = D[o + (j - 1) * d + i - 1];
        for (i64 k = 1; k <= j - 1; ++k) t -= D[o + (k - 1) * d + i - 1] * D[o + (k - 1) * d + j - 1];
        D[o + (j - 1) * d + i - 1] = t / ljj;
      }
    }
    o += d * d;
  }
  return true;
}
template <class T>
void solve_diagonal_blocks(double* y, const T* D, const i64* dims, i64 nb, const double* x) {
  i64 o = 0, p = 0;
  for (i64 b = 0; b < nb; ++b) {
    i64 d = dims[b];
    if (y != x) for (i64 i = 1; i <= d; ++i) y[p + i - 1] = x[p + i - 1];
    for (i64 j = 1; j <= d; ++j) {
      double yj = y[p + j - 1] / (double)D[o + (j - 1) * d + j - 1];
      y[p + j - 1] = yj;
      for (i64 i = j + 1; i <= d; ++i) y[p + i - 1] -= (double)D[o + (j - 1) * d + i - 1] * yj;
    }
    for (i64 j = d; j >= 1; --j) {
      double t = y[p + j - 1];
      for (i64 i = j + 1; i <= d; ++i) t -= (double)D[o + (j - 1) * d + i - 1] * y[p + i - 1];
      y[p + j - 1] = t / (double)D[o + (j - 1) * d + j - 1];
    }
    o += d * d;
    p += d;
  }
}

// makesparseindices (src/SparseBlockLinearSystem.jl:233-282) for the retained storage R (square, lower-triangle blocks,
// `indices` = the transpose of indicestransposed). Outputs the CSC colptr / rowval and the scatter map (1-based).
struct SparseIdx { IV colptr, rowval, map; i64 m = 0, n = 0; };
SparseIdx makesparseindices(const Structure& st, const RLayout& L, bool symmetrify) {
  i64 nb = st.nrblocks;
  // indices = sparse(indicestransposed'): CSC over R column blocks, rows = R row blocks (>= column), nzval = data start
  IV ind_colptr(nb + 1, 0), ind_rowval(L.it_rowval.len()), ind_nzval(L.it_rowval.len());
  {
    IV cnt(nb + 1, 0);
    for (i64 brow = 1; brow <= nb; ++brow)
      for (i64 k = L.it_colptr(brow); k <= L.it_colptr(brow + 1) - 1; ++k) cnt(L.it_rowval(k) + 1) += 1;
    ind_colptr(1) = 1;
    for (i64 c = 1; c <= nb; ++c) ind_colptr(c + 1) = ind_colptr(c) + cnt(c + 1);
    IV pos = ind_colptr;
    for (i64 brow = 1; brow <= nb; ++brow)   // ascending brow keeps rows sorted within each column
      for (i64 k = L.it_colptr(brow); k <= L.it_colptr(brow + 1) - 1; ++k) {
        i64 bcol = L.it_rowval(k);
        ind_rowval(pos(bcol)) = brow; ind_nzval(pos(bcol)) = L.it_nzval(k); pos(bcol) += 1;
      }
  }
  i64 diagspace = 0;   // diagonalblockspace (:217-231)
  for (i64 col = 1; col <= nb; ++col) {
    i64 ind = ind_colptr(col);
    if (ind_colptr(col + 1) > ind) {
      i64 row = ind_rowval(ind);
      if (!(row >= col)) arg_error("SparseBlockLinearSystem must be lower triangular for symmetrification");
      if (row == col) diagspace += st.r_dims(row) * st.r_dims(row);
    }
  }
  i64 nzvals = symmetrify ? L.length * 2 - diagspace : L.length;
  SparseIdx S;
  S.rowval = IV(nzvals); S.map = IV(nzvals);
  IV startrow(nb + 1);
  startrow(1) = 1;
  for (i64 b = 1; b <= nb; ++b) startrow(b + 1) = startrow(b) + st.r_dims(b);
  S.colptr = IV(startrow(nb + 1));
  i64 ind = 1, col = 1;
  S.colptr(1) = 1;
  for (i64 col_ = 1; col_ <= nb; ++col_) {
    i64 colblocksize = st.r_dims(col_);
    i64 lo_first = ind_colptr(col_), lo_last = ind_colptr(col_ + 1) - 1;
    bool has_lower = lo_last >= lo_first;
    i64 up_first = 1, up_last = 0;
    if (symmetrify) {
      up_first = L.it_colptr(col_);
      up_last = L.it_colptr(col_ + 1) - 1 - ((has_lower && ind_rowval(lo_first) == col_) ? 1 : 0);
    }
    for (i64 innercol = 0; innercol <= colblocksize - 1; ++innercol) {
      for (i64 r = up_first; r <= up_last; ++r) {
        i64 row = L.it_rowval(r), s = startrow(row), c = st.r_dims(row), v = L.it_nzval(r) + innercol;
        for (i64 i = 0; i <= c - 1; ++i) { S.rowval(ind) = s + i; S.map(ind) = v; ind += 1; v += colblocksize; }
      }
      for (i64 r = lo_first; r <= lo_last; ++r) {
        i64 row = ind_rowval(r), s = startrow(row), c = st.r_dims(row), v = ind_nzval(r) + innercol * c;
        for (i64 i = 0; i <= c - 1; ++i) { S.rowval(ind) = s + i; S.map(ind) = v + i; ind += 1; }
      }
      col += 1;
      S.colptr(col) = ind;
    }
  }
  S.m = startrow(nb + 1) - 1;
  S.n = col - 1;
  return S;
}

}  // namespace

// ----------------------------------------------------------------------------------------------------------------------
// Block-Jacobi PCG on the reduced system S x = g (no counterpart in the reference: the CPU restatement of the device
// solve, used as its checker and its timed CPU baseline). S: the upper triangle on the pattern; the symmetric matrix's
// rows are gathered from it through an index built once per call. FP64 vectors; the block-Jacobi blocks are S's
// diagonal blocks factored by factor_diagonal_blocks (src/diagonal_blocks.jl:6-29). Same stopping rule as the device:
// recursive residual, then an explicit residual with restarts while it is above tol.
// ----------------------------------------------------------------------------------------------------------------------
template <class T>
int pcg_solve(const Structure& st, const Pattern& P, const T* S, const double* g, double* x, double tol, i64 maxit, int nthreads,
              i64* iters_out, double* rel_out) {
  const i64 nr = st.nr, nrb = st.nrblocks;
  // symmetric rows: row i takes (j, pos) for every stored upper entry (i, j) and (j, i)
  std::vector<i64> cnt(nr + 1, 0);
  for (i64 j = 1; j <= nr; ++j)
    for (i64 q = P.S_colptr(j); q <= P.S_colptr(j + 1) - 1; ++q) {
      const i64 i = P.S_rowval(q);
      if (i > j) continue;
      cnt[i] += 1;
      if (i < j) cnt[j] += 1;
    }
  std::vector<i64> rp(nr + 1, 0);
  for (i64 i = 0; i < nr; ++i) rp[i + 1] = rp[i] + cnt[i + 1];
  std::vector<i64> rc(rp[nr]), rq(rp[nr]), fill(rp.begin(), rp.end() - 1);
  for (i64 j = 1; j <= nr; ++j)
    for (i64 q = P.S_colptr(j); q <= P.S_colptr(j + 1) - 1; ++q) {
      const i64 i = P.S_rowval(q);
      if (i > j) continue;
      rc[fill[i - 1]] = j - 1; rq[fill[i - 1]] = q - 1; fill[i - 1] += 1;
      if (i < j) { rc[fill[j - 1]] = i - 1; rq[fill[j - 1]] = q - 1; fill[j - 1] += 1; }
    }
  auto spmv = [&](const double* v, double* y) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (i64 i = 0; i < nr; ++i) {
      double a = 0.0;
      for (i64 e = rp[i]; e < rp[i + 1]; ++e) a += (double)S[rq[e]] * v[rc[e]];
      y[i] = a;
    }
  };
  // block-Jacobi: S's diagonal blocks, mirrored, factored
  std::vector<double> D;
  std::vector<i64> doff(nrb + 1, 0), dims(nrb);
  for (i64 r = 1; r <= nrb; ++r) { dims[r - 1] = st.r_dims(r); doff[r] = doff[r - 1] + dims[r - 1] * dims[r - 1]; }
  D.assign(doff[nrb], 0.0);
  for (i64 r = 1; r <= nrb; ++r) {
    const i64 d = dims[r - 1], ro = st.boffsets_r(r);
    for (i64 w = 0; w < d; ++w)
      for (i64 a = 0; a < d; ++a) {
        const i64 lo = std::min(a, w), hi = std::max(a, w);
        const i64 col = ro + hi;
        // the entry (ro + lo, col): the diagonal block's rows are contiguous in column col, ending at (col, col)
        D[doff[r - 1] + w * d + a] = (double)S[P.diag_inds(col) - (hi - lo) - 1];
      }
  }
  if (!factor_diagonal_blocks<double>(D.data(), dims.data(), nrb)) return ORC_NOT_PD;
  std::vector<double> r(nr), z(nr), p(nr), q(nr);
  auto precond = [&](const double* in, double* out) { solve_diagonal_blocks<double>(out, D.data(), dims.data(), nrb, in); };
  auto dot = [&](const double* a, const double* b) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static) num_threads(nthreads)
    for (i64 i = 0; i < nr; ++i) s += a[i] * b[i];
    return s;
  };
  const double gg = dot(g, g);
  if (gg == 0.0) { for (i64 i = 0; i < nr; ++i) x[i] = 0.0; *iters_out = 0; *rel_out = 0.0; return ORC_OK; }
  const double t2 = tol * tol * gg;
  i64 iters = 0;
  double rel = INFINITY;
  for (int restart = 0; restart < 4; ++restart) {
    spmv(x, q.data());
    for (i64 i = 0; i < nr; ++i) r[i] = g[i] - q[i];
    precond(r.data(), z.data());
    p = z;
    double rz = dot(r.data(), z.data()), rr = dot(r.data(), r.data());
    while (rr > t2 && iters < maxit) {
      spmv(p.data(), q.data());
      const double alpha = rz / dot(p.data(), q.data());
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (i64 i = 0; i < nr; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
      precond(r.data(), z.data());
      const double rzn = dot(r.data(), z.data());
      rr = dot(r.data(), r.data());
      ++iters;
      if (!(rr > t2)) break;
      const double beta = rzn / rz;
      rz = rzn;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (i64 i = 0; i < nr; ++i) p[i] = z[i] + beta * p[i];
    }
    spmv(x, q.data());
    for (i64 i = 0; i < nr; ++i) r[i] = g[i] - q[i];
    rel = std::sqrt(dot(r.data(), r.data()) / gg);
    if (rel <= tol || iters >= maxit || !std::isfinite(rel)) break;
  }
  *iters_out = iters;
  *rel_out = rel;
  return rel <= tol ? ORC_OK : 2;
}

// ======================================================================================================================
// extern "C" boundary: 0-based integers, status codes (0 ok, 1 singular/not positive definite, < 0 argument errors)
// ======================================================================================================================
struct OrcStructure { Structure st; };
struct OrcPattern { Pattern P; RLayout L; };
struct OrcWork { Work<double>* w64 = nullptr; Work<float>* w32 = nullptr; ~OrcWork() { delete w64; delete w32; } };
struct OrcQR { QRStructure q; };

static thread_local std::string g_err;
static int fail(const BlsError& e) { g_err = e.what(); return e.code; }

#define ORC_TRY(...) try { __VA_ARGS__ } catch (const BlsError& e) { return fail(e); } catch (const std::exception& e) { g_err = e.what(); return ORC_EINVAL; }

static std::vector<std::vector<i64>> csr_lists_1based(i64 K, const i64* ptr, const i64* idx) {
  std::vector<std::vector<i64>> out((size_t)K);
  for (i64 k = 0; k < K; ++k)
    for (i64 p = ptr[k]; p < ptr[k + 1]; ++p) out[k].push_back(idx[p] + 1);
  return out;
}
static IV iv_from(const i64* a, i64 n) { IV v(n); for (i64 i = 0; i < n; ++i) v.v[i] = a[i]; return v; }
static i64 put(i64* out, const std::vector<i64>& v, i64 shift) {
  if (out) for (size_t i = 0; i < v.size(); ++i) out[i] = v[i] + shift;
  return (i64)v.size();
}

// reduced_mul! (src/qr_reduced.jl:159-192): y = J~ v, accumulated per row in the order of the table's entries and columns
template <class T>
void reduced_mul(double* y, i64 ny, const double* v, i64 nv, const T* F, const QRStructure& q) {
  const Structure& st = q.schur;
  const i64 nred = q.reduced_offsets(q.ntables + 1) - 1;
  if (ny != nred) dim_error("y has length " + std::to_string(ny) + ", expected " + std::to_string(nred));
  if (nv != st.nr) dim_error("v has length " + std::to_string(nv) + ", expected " + std::to_string(st.nr));
  for (i64 t = 1; t <= q.ntables; ++t) {
    const i64 M = q.table_nrows(t), top = q.table_top(t), off = q.raw_offsets(t), yo = q.reduced_offsets(t), n = M - top;
    for (i64 i = 0; i <= n - 1; ++i) y[yo + i - 1] = 0.0;
    for (i64 u = q.table_ptr(t); u <= q.table_ptr(t + 1) - 1; ++u) {
      const i64 r = q.entry_retained(u), ro = st.boffsets_r(r), cb = off + (q.entry_col(u) - 1) * M + top;
      for (i64 j = 1; j <= st.r_dims(r); ++j) {
        const double vj = v[ro + j - 2];
        const i64 c0 = cb + (j - 1) * M;
        for (i64 i = 0; i <= n - 1; ++i) y[yo + i - 1] += (double)F[c0 + i - 1] * vj;
      }
    }
  }
}

// reduced_tmul! (src/qr_reduced.jl:194-223): g = J~' w, per retained column the runs' dot products (dot_run, FP64)
template <class T>
void reduced_tmul(double* g, i64 ng, const double* w, i64 nw, const T* F, const QRStructure& q) {
  const Structure& st = q.schur;
  const i64 nred = q.reduced_offsets(q.ntables + 1) - 1;
  if (ng != st.nr) dim_error("g has length " + std::to_string(ng) + ", expected " + std::to_string(st.nr));
  if (nw != nred) dim_error("w has length " + std::to_string(nw) + ", expected " + std::to_string(nred));
  for (i64 r = 1; r <= st.nrblocks; ++r) {
    const i64 ro = st.boffsets_r(r), dr = st.r_dims(r);
    for (i64 j = 0; j <= dr - 1; ++j) g[ro + j - 1] = 0.0;
    for (i64 k = q.retained_ptr(r); k <= q.retained_ptr(r + 1) - 1; ++k) {
      const i64 u = q.retained_entry(k), t = q.entry_table(u), M = q.table_nrows(t), top = q.table_top(t);
      const i64 cb = q.raw_offsets(t) + (q.entry_col(u) - 1) * M + top, wo = q.reduced_offsets(t);
      for (i64 j = 1; j <= dr; ++j) {
        double acc = 0.0;
        for (i64 i = 0; i <= M - top - 1; ++i) acc += (double)F[cb + (j - 1) * M + i - 1] * w[wo + i - 1];
        g[ro + j - 2] += acc;
      }
    }
  }
}

// reduced_residual! (src/qr_reduced.jl:227-243): r~ in the row order of the reduced problem
void reduced_residual(double* rt, i64 n_rt, const double* Fr, const QRStructure& q) {
  const i64 nred = q.reduced_offsets(q.ntables + 1) - 1;
  if (n_rt != nred) dim_error("rt has length " + std::to_string(n_rt) + ", expected " + std::to_string(nred));
  for (i64 t = 1; t <= q.ntables; ++t) {
    const i64 M = q.table_nrows(t), top = q.table_top(t), cb = q.residual_offsets(t) + top, ro = q.reduced_offsets(t);
    for (i64 i = 0; i <= M - top - 1; ++i) rt[ro + i - 1] = Fr[cb + i - 1];
  }
}

// reduced_jacobian!(Jt::AbstractMatrix, rt, ws) (src/qr_reduced.jl:245-272): J~ densely, column-major nrows x ncols
template <class T>
void reduced_jacobian_dense(T* Jt, i64 nrows, i64 ncols, double* rt, i64 n_rt, const T* F, const double* Fr, const QRStructure& q) {
  const Structure& st = q.schur;
  const i64 nred = q.reduced_offsets(q.ntables + 1) - 1;
  if (nrows != nred || ncols != st.nr)
    dim_error("Jt has size (" + std::to_string(nrows) + ", " + std::to_string(ncols) + "), expected (" + std::to_string(nred) + ", " +
              std::to_string(st.nr) + ")");
  if (n_rt != nred) dim_error("rt has length " + std::to_string(n_rt) + ", expected " + std::to_string(nred));
  for (i64 k = 0; k < nrows * ncols; ++k) Jt[k] = T(0);
  reduced_residual(rt, n_rt, Fr, q);
  for (i64 t = 1; t <= q.ntables; ++t) {
    const i64 M = q.table_nrows(t), top = q.table_top(t), off = q.raw_offsets(t), yo = q.reduced_offsets(t);
    for (i64 u = q.table_ptr(t); u <= q.table_ptr(t + 1) - 1; ++u) {
      const i64 r = q.entry_retained(u), ro = st.boffsets_r(r), cb = off + (q.entry_col(u) - 1) * M + top;
      for (i64 j = 1; j <= st.r_dims(r); ++j)
        for (i64 i = 0; i <= M - top - 1; ++i) Jt[(yo + i - 1) + nrows * (ro + j - 2)] = F[cb + (j - 1) * M + i - 1];
    }
  }
}

// reduced_column_height (src/qr_reduced.jl:274-282)
i64 reduced_column_height(const QRStructure& q, i64 r) {
  i64 h = 0;
  for (i64 k = q.retained_ptr(r); k <= q.retained_ptr(r + 1) - 1; ++k) {
    const i64 t = q.entry_table(q.retained_entry(k));
    h += q.table_nrows(t) - q.table_top(t);
  }
  return h;
}

// build_reduced_jacobian_pattern (src/qr_reduced.jl:284-310), 1-based colptr (nr + 1) and rowval
void reduced_jacobian_pattern(const QRStructure& q, IV& colptr, IV& rowval) {
  const Structure& st = q.schur;
  colptr = IV(st.nr + 1);
  colptr(1) = 1;
  for (i64 r = 1; r <= st.nrblocks; ++r) {
    const i64 h = reduced_column_height(q, r), ro = st.boffsets_r(r);
    for (i64 j = 0; j <= st.r_dims(r) - 1; ++j) colptr(ro + j + 1) = colptr(ro + j) + h;
  }
  rowval = IV(colptr(st.nr + 1) - 1);
  for (i64 r = 1; r <= st.nrblocks; ++r)
    for (i64 j = 0; j <= st.r_dims(r) - 1; ++j) {
      i64 p = colptr(st.boffsets_r(r) + j);
      for (i64 k = q.retained_ptr(r); k <= q.retained_ptr(r + 1) - 1; ++k) {
        const i64 t = q.entry_table(q.retained_entry(k));
        for (i64 i = 0; i <= q.table_nrows(t) - q.table_top(t) - 1; ++i) { rowval(p) = q.reduced_offsets(t) + i; p += 1; }
      }
    }
}

// check_reduced_jacobian_pattern (src/qr_reduced.jl:312-334) on a 1-based CSC
void check_reduced_jacobian_pattern(i64 nrows, i64 ncols, const IV& colptr, const IV& rowval, const QRStructure& q) {
  const Structure& st = q.schur;
  const i64 nred = q.reduced_offsets(q.ntables + 1) - 1;
  if (nrows != nred || ncols != st.nr)
    dim_error("Jt has size (" + std::to_string(nrows) + ", " + std::to_string(ncols) + "), expected (" + std::to_string(nred) + ", " +
              std::to_string(st.nr) + ")");
  for (i64 r = 1; r <= st.nrblocks; ++r) {
    const i64 h = reduced_column_height(q, r);
    for (i64 c = st.boffsets_r(r); c <= st.boffsets_r(r) + st.r_dims(r) - 1; ++c) {
      if (colptr(c + 1) - colptr(c) != h)
        arg_error("Jt does not have the pattern of build_reduced_jacobian_pattern: column " + std::to_string(c) + " stores " +
                  std::to_string(colptr(c + 1) - colptr(c)) + " entries, expected " + std::to_string(h));
      i64 p = colptr(c);
      for (i64 k = q.retained_ptr(r); k <= q.retained_ptr(r + 1) - 1; ++k) {
        const i64 t = q.entry_table(q.retained_entry(k));
        const i64 n = q.table_nrows(t) - q.table_top(t);
        if (!(n == 0 || rowval(p) == q.reduced_offsets(t)))
          arg_error("Jt does not have the pattern of build_reduced_jacobian_pattern: column " + std::to_string(c) + " stores row " +
                    std::to_string(rowval(p)) + ", expected " + std::to_string(q.reduced_offsets(t)));
        p += n;
      }
    }
  }
}

// reduced_jacobian!(Jt::SparseMatrixCSC, rt, ws) (src/qr_reduced.jl:336-370): J~ into nzval of the pattern
template <class T>
void reduced_jacobian_sparse(i64 nrows, i64 ncols, const IV& colptr, const IV& rowval, T* nzval, double* rt, i64 n_rt, const T* F,
                             const double* Fr, const QRStructure& q) {
  const Structure& st = q.schur;
  check_reduced_jacobian_pattern(nrows, ncols, colptr, rowval, q);
  reduced_residual(rt, n_rt, Fr, q);
  for (i64 r = 1; r <= st.nrblocks; ++r) {
    const i64 ro = st.boffsets_r(r), dr = st.r_dims(r);
    i64 p = 0;
    for (i64 k = q.retained_ptr(r); k <= q.retained_ptr(r + 1) - 1; ++k) {
      const i64 u = q.retained_entry(k), t = q.entry_table(u), M = q.table_nrows(t), top = q.table_top(t), n = M - top;
      const i64 cb = q.raw_offsets(t) + (q.entry_col(u) - 1) * M + top;
      for (i64 j = 0; j <= dr - 1; ++j) {
        const i64 qq = colptr(ro + j) + p, c0 = cb + j * M;
        for (i64 i = 0; i <= n - 1; ++i) nzval[qq + i - 1] = F[c0 + i - 1];
      }
      p += n;
    }
  }
}

// find_in_column (src/schur_structure.jl:355-361) on a 1-based CSC: the index of `row` in column j, 0 if absent
static i64 find_in_column_1(const IV& S_colptr, const IV& S_rowval, i64 row, i64 j) {
  i64 lo = S_colptr(j), hi = S_colptr(j + 1) - 1;
  // searchsortedfirst over rowval[lo:hi]
  i64 a = lo, b = hi + 1;
  while (a < b) {
    const i64 mid = (a + b) / 2;
    if (S_rowval(mid) < row) a = mid + 1;
    else b = mid;
  }
  return (a <= hi && S_rowval(a) == row) ? a : 0;
}

// build_r_to_s_map(R_sparse, S_sparse) (src/schur_structure.jl:336-353), 1-based
IV r_to_s_map_csc(i64 ncols, const IV& R_colptr, const IV& R_rowval, const IV& S_colptr, const IV& S_rowval) {
  IV r_to_s(R_colptr(ncols + 1) - 1, 0);
  i64 pos = 1;
  for (i64 j = 1; j <= ncols; ++j)
    for (i64 k = R_colptr(j); k <= R_colptr(j + 1) - 1; ++k) {
      const i64 i = R_rowval(k), s_k = find_in_column_1(S_colptr, S_rowval, i, j);
      if (s_k == 0) arg_error("R entry (" + std::to_string(i) + ", " + std::to_string(j) + ") is not present in the sparsity pattern of S");
      r_to_s(pos++) = s_k;
    }
  return r_to_s;
}

// build_r_to_s_map(R_sys, S_sparse, boffsets_r) (src/schur_structure.jl:363-397), 1-based
IV r_to_s_map_blocks_csc(i64 nb, const IV& sizes, const IV& it_colptr, const IV& it_rowval, const IV& it_nzval, i64 data_len,
                         const IV& S_colptr, const IV& S_rowval, const IV& boffsets_r) {
  IV r_to_s(data_len, 0);
  for (i64 brow = 1; brow <= nb; ++brow)
    for (i64 k = it_colptr(brow); k <= it_colptr(brow + 1) - 1; ++k) {
      const i64 bcol = it_rowval(k), data_start = it_nzval(k), drow = sizes(brow), dcol = sizes(bcol);
      if (brow == bcol) {
        for (i64 col = 1; col <= dcol; ++col) {
          const i64 scol = boffsets_r(brow) + col - 1;
          for (i64 row = 1; row <= col; ++row) {
            const i64 srow = boffsets_r(brow) + row - 1, s_k = find_in_column_1(S_colptr, S_rowval, srow, scol);
            if (s_k == 0)
              arg_error("Entry (" + std::to_string(srow) + ", " + std::to_string(scol) + ") of a diagonal block of R is not present in the sparsity pattern of S");
            r_to_s(data_start + (col - 1) * drow + row - 1) = s_k;
          }
        }
      } else if (brow > bcol) {
        for (i64 col = 1; col <= dcol; ++col) {
          const i64 srow = boffsets_r(bcol) + col - 1;
          for (i64 row = 1; row <= drow; ++row) {
            const i64 scol = boffsets_r(brow) + row - 1, s_k = find_in_column_1(S_colptr, S_rowval, srow, scol);
            if (s_k == 0) arg_error("Entry (" + std::to_string(srow) + ", " + std::to_string(scol) + ") of R is not present in the sparsity pattern of S");
            r_to_s(data_start + (col - 1) * drow + row - 1) = s_k;
          }
        }
      }
    }
  return r_to_s;
}

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int orc_structure_from_description(i64 n, const i64* blocksizes, i64 K, const i64* rb_ptr, const i64* rb_idx,
                                   const uint8_t* eliminated, i64 nchunks, i64 min_work, OrcStructure** out) {
  ORC_TRY({
    std::vector<bool> el((size_t)n);
    for (i64 i = 0; i < n; ++i) el[i] = eliminated[i] != 0;
    auto* o = new OrcStructure();
    o->st = structure_from_description(iv_from(blocksizes, n), csr_lists_1based(K, rb_ptr, rb_idx), el, nullptr, nchunks, min_work);
    *out = o;
    return ORC_OK;
  })
}

int orc_structure_positional(i64 nrb, const i64* r_dims, i64 neb, const i64* e_dims, const i64* cp_ptr, const i64* cp_idx,
                             i64 nchunks, i64 min_work, OrcStructure** out) {
  ORC_TRY({
    auto lists = csr_lists_1based(neb, cp_ptr, cp_idx);
    std::vector<IV> coup;
    for (auto& l : lists) { IV v; v.v = l; coup.push_back(v); }
    auto* o = new OrcStructure();
    o->st = make_structure(iv_from(r_dims, nrb), iv_from(e_dims, neb), coup, nchunks, min_work, nullptr, {});
    *out = o;
    return ORC_OK;
  })
}

void orc_structure_free(OrcStructure* s) { delete s; }

// Field getter: returns the length; copies into `out` when it is not null. Index-valued fields are 0-based.
i64 orc_structure_field(OrcStructure* o, const char* name, i64* out) {
  const Structure& st = o->st;
  std::string f(name);
  if (f == "nr") { if (out) out[0] = st.nr; return 1; }
  if (f == "nrblocks") { if (out) out[0] = st.nrblocks; return 1; }
  if (f == "neblocks") { if (out) out[0] = st.neblocks; return 1; }
  if (f == "max_coupled_dim") { if (out) out[0] = st.max_coupled_dim; return 1; }
  if (f == "r_dims") return put(out, st.r_dims.v, 0);
  if (f == "e_dims") return put(out, st.e_dims.v, 0);
  if (f == "boffsets_r") return put(out, st.boffsets_r.v, -1);
  if (f == "boffsets_e") return put(out, st.boffsets_e.v, -1);
  if (f == "eoffsets") return put(out, st.eoffsets.v, -1);
  if (f == "eliminated_ptr") return put(out, st.eliminated_ptr.v, -1);
  if (f == "entry_retained") return put(out, st.entry_retained.v, -1);
  if (f == "coffsets") return put(out, st.coffsets.v, -1);
  if (f == "order") return put(out, st.order.v, -1);
  if (f == "retained_pairs") {
    std::vector<i64> v;
    for (auto& p : st.retained_pairs) { v.push_back(p.first); v.push_back(p.second); }
    return put(out, v, -1);
  }
  if (f == "chunks") {   // per run, per chunk: (first, stop) as a 0-based half-open range
    std::vector<i64> v;
    for (auto& run : st.chunks) for (auto& c : run) { v.push_back(c.first - 1); v.push_back(c.last); }
    return put(out, v, 0);
  }
  if (f == "e_run_sizes") return put(out, st.e_runs.size, 0);
  if (f == "e_run_lengths") return put(out, st.e_runs.len, 0);
  return -1;
}

int orc_expand_block_perm(i64 n, const i64* perm, const i64* sizes, i64* out) {
  ORC_TRY({
    IV p = iv_from(perm, n);
    for (auto& x : p.v) x += 1;
    IV s = expand_block_perm(p, iv_from(sizes, n));
    put(out, s.v, -1);
    return ORC_OK;
  })
}

int orc_sort_schur_blocks(i64 n, const uint8_t* is_elim, const i64* sizes, const i64* cp_ptr, const i64* cp_idx, i64* out) {
  ORC_TRY({
    std::vector<bool> el((size_t)n);
    for (i64 i = 0; i < n; ++i) el[i] = is_elim[i] != 0;
    IV o = sort_schur_blocks(el, iv_from(sizes, n), csr_lists_1based(n, cp_ptr, cp_idx));
    put(out, o.v, -1);
    return ORC_OK;
  })
}

int orc_schur_pattern(OrcStructure* o, i64 nextra, const i64* extra, OrcPattern** out) {
  ORC_TRY({
    std::vector<std::pair<i64, i64>> ex;
    for (i64 i = 0; i < nextra; ++i) ex.push_back({extra[2 * i] + 1, extra[2 * i + 1] + 1});
    auto* p = new OrcPattern();
    p->P = build_schur_pattern(o->st, ex);
    p->L = r_layout(o->st, p->P);
    *out = p;
    return ORC_OK;
  })
}
void orc_pattern_free(OrcPattern* p) { delete p; }

i64 orc_pattern_field(OrcPattern* o, const char* name, i64* out) {
  const Pattern& P = o->P;
  std::string f(name);
  if (f == "block_colptr") return put(out, P.block_colptr.v, -1);
  if (f == "block_rowval") return put(out, P.block_rowval.v, -1);
  if (f == "block_row_offsets") return put(out, P.block_row_offsets.v, 0);
  if (f == "col_heights") return put(out, P.col_heights.v, 0);
  if (f == "S_colptr") return put(out, P.S_colptr.v, -1);
  if (f == "S_rowval") return put(out, P.S_rowval.v, -1);
  if (f == "diag_inds") return put(out, P.diag_inds.v, -1);
  if (f == "R_block_start") return put(out, o->L.it_nzval.v, -1);   // per block in block_colptr order (R row block = column)
  if (f == "R_length") { if (out) out[0] = o->L.length; return 1; }
  return -1;
}

// r_to_s map, 0-based, -1 where unmapped (the reference's 0)
int orc_r_to_s_map(OrcStructure* o, OrcPattern* p, i64* out) {
  ORC_TRY({
    IV m = build_r_to_s_map(o->st, p->P, p->L);
    put(out, m.v, -1);
    return ORC_OK;
  })
}

// symmetrifyfull!(mat, bsm, blocks) (src/SparseBlockLinearSystem.jl:299-341) for a block-square system given by its
// block sizes and indicestransposed (a CSC over block rows r: rows it_rowval = block columns c, values it_nzval = the
// 0-based start of block (r, c) in data, column-major blocksizes[r] x blocksizes[c]). blocks: 0-based block list, in
// the order the blocks take in mat, or NULL for all blocks in order (nblocks is then ignored). mat: m x m, column-major.
int orc_symmetrify_full(i64 nb, const i64* blocksizes, const i64* it_colptr, const i64* it_rowval, const i64* it_nzval,
                        const double* data, const i64* blocks, i64 nblocks, double* mat, i64 m) {
  ORC_TRY({
    IV lengths(nb, 0), starts(nb, 0);   // 1-based starts; 0 marks a block left out
    if (!blocks) {
      i64 cur = 1;
      for (i64 b = 1; b <= nb; ++b) { lengths(b) = blocksizes[b - 1]; starts(b) = cur; cur += blocksizes[b - 1]; }
    } else {
      if (nblocks == 0) {
        if (m != 0) dim_error("Target matrix has size (" + std::to_string(m) + ", " + std::to_string(m) + "), expected (0, 0)");
        return ORC_OK;
      }
      for (i64 i = 0; i < nblocks; ++i)
        if (!(blocks[i] >= 0 && blocks[i] < nb)) arg_error("BoundsError: block " + std::to_string(blocks[i] + 1) + " of " + std::to_string(nb));
      for (i64 i = 0; i < nblocks; ++i) {
        const i64 b = blocks[i] + 1;
        if (lengths(b) != 0) arg_error("Block " + std::to_string(b) + " is listed more than once");
        lengths(b) = blocksizes[b - 1];
      }
      i64 cur = 1;
      for (i64 i = 0; i < nblocks; ++i) { starts(blocks[i] + 1) = cur; cur += blocksizes[blocks[i]]; }
    }
    i64 total = 0;
    for (i64 b = 1; b <= nb; ++b) total += lengths(b);
    if (total != m)
      dim_error("Target matrix has size (" + std::to_string(m) + ", " + std::to_string(m) + "), expected (" + std::to_string(total) + ", " +
                std::to_string(total) + ")");
    for (i64 q = 0; q < m * m; ++q) mat[q] = 0.0;
    // findnz(indicestransposed): block columns r of the transpose in order, then its rows c
    for (i64 r = 1; r <= nb; ++r)
      for (i64 k = it_colptr[r - 1]; k < it_colptr[r]; ++k) {
        const i64 c = it_rowval[k] + 1, index = it_nzval[k];
        const i64 cs = starts(c);
        if (cs == 0) continue;
        const i64 rs = starts(r);
        if (rs == 0) continue;
        const i64 r_ = lengths(r), c_ = lengths(c);
        for (i64 cc = 0; cc < c_; ++cc)
          for (i64 rr = 0; rr < r_; ++rr) {
            const double v = data[index + rr + cc * r_];
            mat[(rs - 1 + rr) + m * (cs - 1 + cc)] = v;
            if (r != c) mat[(cs - 1 + cc) + m * (rs - 1 + rr)] = v;
          }
      }
    return ORC_OK;
  })
}

// makesparseindices + sparse_with_map of the retained storage: colptr (n+1), rowval, map (0-based)
i64 orc_sparse_indices(OrcStructure* o, OrcPattern* p, int symmetric, i64* colptr, i64* rowval, i64* map) {
  SparseIdx S;
  try { S = makesparseindices(o->st, p->L, symmetric != 0); } catch (const BlsError& e) { g_err = e.what(); return -1; }
  put(colptr, S.colptr.v, -1);
  put(rowval, S.rowval.v, -1);
  put(map, S.map.v, -1);
  return S.map.len();
}

int orc_work_new(OrcStructure* o, i64 nchunks, int f32, OrcWork** out) {
  ORC_TRY({
    auto* w = new OrcWork();
    if (f32) w->w32 = make_work<float>(o->st, nchunks);
    else w->w64 = make_work<double>(o->st, nchunks);
    *out = w;
    return ORC_OK;
  })
}
void orc_work_free(OrcWork* w) { delete w; }

i64 orc_work_field(OrcWork* w, const char* name, i64* out) {
  std::string f(name);
  const IV* rp = w->w64 ? &w->w64->retained_ptr : &w->w32->retained_ptr;
  const IV* re = w->w64 ? &w->w64->retained_entry : &w->w32->retained_entry;
  const IV* ee = w->w64 ? &w->w64->entry_eliminated : &w->w32->entry_eliminated;
  const auto& cc = w->w64 ? w->w64->col_chunks : w->w32->col_chunks;
  if (f == "retained_ptr") return put(out, rp->v, -1);
  if (f == "retained_entry") return put(out, re->v, -1);
  if (f == "entry_eliminated") return put(out, ee->v, -1);
  if (f == "col_chunks") {
    std::vector<i64> v;
    for (auto& c : cc) { v.push_back(c.first - 1); v.push_back(c.last); }
    return put(out, v, 0);
  }
  return -1;
}

// E_inv and z caches of the last reduction (for tests)
void orc_work_caches(OrcWork* w, void* E_inv, double* z) {
  if (w->w64) { std::memcpy(E_inv, w->w64->E_inv_data.data(), 8 * w->w64->E_inv_data.size()); std::memcpy(z, w->w64->z_data.data(), 8 * w->w64->z_data.size()); }
  else { std::memcpy(E_inv, w->w32->E_inv_data.data(), 4 * w->w32->E_inv_data.size()); std::memcpy(z, w->w32->z_data.data(), 8 * w->w32->z_data.size()); }
}

#define ORC_TYPED(SUFFIX, T, WMEMBER)                                                                                          \
  int orc_reset_schur_sparse_##SUFFIX(OrcStructure* o, OrcPattern* p, T* nzval, const T* R_data, const double* scaling_r,     \
                                      double lambda, const double* s_r) {                                                      \
    ORC_TRY({                                                                                                                   \
      IV m = build_r_to_s_map(o->st, p->P, p->L);                                                                               \
      reset_sparse<T>(nzval, p->P.S_rowval.len(), R_data, m, p->P.diag_inds, scaling_r, o->st.nr, lambda, s_r, &p->P.S_colptr, \
                      &p->P.S_rowval);                                                                                          \
      return ORC_OK;                                                                                                            \
    })                                                                                                                          \
  }                                                                                                                             \
  int orc_reset_schur_dense_##SUFFIX(OrcStructure* o, T* S, const T* R, const double* scaling_r, double lambda,              \
                                     const double* s_r) {                                                                       \
    ORC_TRY({ reset_dense<T>(S, R, scaling_r, o->st.nr, lambda, s_r); return ORC_OK; })                                        \
  }                                                                                                                             \
  int orc_reduce_schur_sparse_##SUFFIX(OrcStructure* o, OrcPattern* p, OrcWork* w, T* nzval, double* g_S, const double* b_r,  \
                                       const double* b_e, const double* scaling_e, double lambda, const T* E, const T* C,      \
                                       const double* s_r, const double* s_e, int nthreads, i64* failed_block) {                \
    ORC_TRY({                                                                                                                   \
      const Structure& st = o->st;                                                                                              \
      i64 ne = 0; for (i64 d : st.e_dims.v) ne += d;                                                                             \
      check_damping(lambda, scaling_e, ne, "scaling_e");                                                                        \
      auto& ws = *w->WMEMBER;                                                                                                   \
      ws.failed_block.store(0);                                                                                                 \
      if (!factor_all<T>(ws, st, E, C, b_e, scaling_e, lambda, s_r, s_e, nthreads)) {                                           \
        *failed_block = ws.failed_block.load();                                                                                 \
        return ORC_NOT_PD;                                                                                                      \
      }                                                                                                                         \
      for (i64 i = 0; i < st.nr; ++i) g_S[i] = s_r ? b_r[i] * s_r[i] : b_r[i];                                                 \
      i64 nk = (i64)ws.col_chunks.size();                                                                                       \
      bool threaded = use_threads(nk, st.entry_retained.len(), st.min_work, nthreads);                                         \
      _Pragma("omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (threaded)")                                      \
      for (i64 k = 0; k < nk; ++k) accumulate_sparse_columns<T>(nzval, g_S, st, C, ws, p->P, ws.col_chunks[k], s_r, s_e);      \
      *failed_block = 0;                                                                                                        \
      return ORC_OK;                                                                                                            \
    })                                                                                                                          \
  }                                                                                                                             \
  int orc_reduce_schur_dense_##SUFFIX(OrcStructure* o, OrcWork* w, T* S, double* g_S, const double* b_r, const double* b_e,   \
                                      const double* scaling_e, double lambda, const T* E, const T* C, const double* s_r,        \
                                      const double* s_e, int nthreads, i64* failed_block) {                                     \
    ORC_TRY({                                                                                                                   \
      const Structure& st = o->st;                                                                                              \
      i64 ne = 0; for (i64 d : st.e_dims.v) ne += d;                                                                             \
      check_damping(lambda, scaling_e, ne, "scaling_e");                                                                        \
      auto& ws = *w->WMEMBER;                                                                                                   \
      ws.failed_block.store(0);                                                                                                 \
      if (!factor_all<T>(ws, st, E, C, b_e, scaling_e, lambda, s_r, s_e, nthreads)) {                                           \
        *failed_block = ws.failed_block.load();                                                                                 \
        return ORC_NOT_PD;                                                                                                      \
      }                                                                                                                         \
      for (i64 i = 0; i < st.nr; ++i) g_S[i] = s_r ? b_r[i] * s_r[i] : b_r[i];                                                 \
      i64 nk = (i64)ws.col_chunks.size();                                                                                       \
      bool threaded = use_threads(nk, st.entry_retained.len(), st.min_work, nthreads);                                         \
      _Pragma("omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (threaded)")                                      \
      for (i64 k = 0; k < nk; ++k) accumulate_dense_columns<T>(S, st.nr, g_S, st, C, ws, ws.col_chunks[k], s_r, s_e);          \
      *failed_block = 0;                                                                                                        \
      return ORC_OK;                                                                                                            \
    })                                                                                                                          \
  }                                                                                                                             \
  int orc_backsubstitute_##SUFFIX(OrcStructure* o, OrcWork* w, double* x_e, const double* x_r, const T* C, const double* s_r, \
                                  const double* s_e, int nthreads) {                                                            \
    ORC_TRY({ backsubstitute<T>(x_e, x_r, o->st, C, *w->WMEMBER, s_r, s_e, nthreads); return ORC_OK; })                       \
  }

ORC_TYPED(f64, double, w64)
ORC_TYPED(f32, float, w32)

// ---- QR ----
int orc_qr_structure_from_description(i64 n, const i64* blocksizes, i64 K, const i64* rb_ptr, const i64* rb_idx,
                                      const i64* rowblocksizes, const uint8_t* eliminated, i64 nchunks, i64 min_work,
                                      OrcQR** out, OrcStructure** st_out) {
  ORC_TRY({
    std::vector<bool> el((size_t)n);
    for (i64 i = 0; i < n; ++i) el[i] = eliminated[i] != 0;
    auto* q = new OrcQR();
    q->q = qr_structure_from_description(iv_from(blocksizes, n), csr_lists_1based(K, rb_ptr, rb_idx), iv_from(rowblocksizes, K), el,
                                         nchunks, min_work);
    *out = q;
    if (st_out) { auto* s = new OrcStructure(); s->st = q->q.schur; *st_out = s; }
    return ORC_OK;
  })
}
int orc_qr_structure_positional(OrcStructure* o, const i64* e_rows, i64 nfree, const i64* free_rows, const i64* free_ptr,
                                const i64* free_idx, i64 nchunks, OrcQR** out) {
  ORC_TRY({
    auto* q = new OrcQR();
    q->q = make_qr_structure(o->st, iv_from(e_rows, o->st.neblocks), iv_from(free_rows, nfree), csr_lists_1based(nfree, free_ptr, free_idx), nchunks);
    q->q.e_rows = iv_from(e_rows, o->st.neblocks);
    q->q.free_rows = iv_from(free_rows, nfree);
    *out = q;
    return ORC_OK;
  })
}
void orc_qr_free(OrcQR* q) { delete q; }

i64 orc_qr_field(OrcQR* o, const char* name, i64* out) {
  const QRStructure& q = o->q;
  std::string f(name);
  if (f == "ntables") { if (out) out[0] = q.ntables; return 1; }
  if (f == "table_nrows") return put(out, q.table_nrows.v, 0);
  if (f == "table_ncols") return put(out, q.table_ncols.v, 0);
  if (f == "table_top") return put(out, q.table_top.v, 0);
  if (f == "table_offsets") return put(out, q.table_offsets.v, -1);
  if (f == "raw_offsets") return put(out, q.raw_offsets.v, -1);
  if (f == "residual_offsets") return put(out, q.residual_offsets.v, -1);
  if (f == "reduced_offsets") return put(out, q.reduced_offsets.v, -1);
  if (f == "table_ptr") return put(out, q.table_ptr.v, -1);
  if (f == "entry_retained") return put(out, q.entry_retained.v, -1);
  if (f == "entry_col") return put(out, q.entry_col.v, -1);
  if (f == "entry_table") return put(out, q.entry_table.v, -1);
  if (f == "retained_ptr") return put(out, q.retained_ptr.v, -1);
  if (f == "retained_entry") return put(out, q.retained_entry.v, -1);
  if (f == "doffsets") return put(out, q.doffsets.v, -1);
  if (f == "e_rows") return put(out, q.e_rows.v, 0);
  if (f == "free_rows") return put(out, q.free_rows.v, 0);
  if (f == "row_table") return put(out, q.row_table.v, -1);
  if (f == "row_first") return put(out, q.row_first.v, -1);
  if (f == "row_nrows") return put(out, q.row_nrows.v, 0);
  if (f == "row_ptr") return put(out, q.row_ptr.v, -1);
  if (f == "row_blocks") return put(out, q.row_blocks.v, -1);
  if (f == "col_chunks") {
    std::vector<i64> v;
    for (auto& c : q.col_chunks) { v.push_back(c.first - 1); v.push_back(c.last); }
    return put(out, v, 0);
  }
  return -1;
}

#define ORC_QR_TYPED(SUFFIX, T)                                                                                                 \
  int orc_reduce_qr_##SUFFIX(OrcQR* o, T* F, double* Fr, const T* Rw, const double* Rr, const double* scaling_e, i64 n_sc,       \
                             double lambda, const double* s, int nthreads, i64* failed_block) {                                   \
    ORC_TRY({ return reduce_qr<T>(o->q, F, Fr, Rw, Rr, scaling_e, n_sc, lambda, s, nthreads, failed_block) ? ORC_OK : ORC_NOT_PD; }) \
  }                                                                                                                               \
  int orc_qr_backsubstitute_##SUFFIX(OrcQR* o, double* x_e, const double* x_r, const T* F, const double* Fr) {                    \
    ORC_TRY({ qr_backsubstitute<T>(x_e, x_r, F, Fr, o->q); return ORC_OK; })                                                     \
  }                                                                                                                               \
  int orc_reduced_normal_sparse_##SUFFIX(OrcQR* o, OrcPattern* p, T* nzval, double* g_S, const T* F, const double* Fr) {         \
    ORC_TRY({ reduced_normal_sparse<T>(nzval, g_S, F, Fr, o->q, p->P); return ORC_OK; })                                         \
  }                                                                                                                               \
  int orc_reduced_normal_dense_##SUFFIX(OrcQR* o, T* S, double* g_S, const T* F, const double* Fr) {                             \
    ORC_TRY({ reduced_normal_dense<T>(S, g_S, F, Fr, o->q); return ORC_OK; })                                                    \
  }                                                                                                                               \
  int orc_reduced_mul_##SUFFIX(OrcQR* o, double* y, i64 ny, const double* v, i64 nv, const T* F) {                              \
    ORC_TRY({ reduced_mul<T>(y, ny, v, nv, F, o->q); return ORC_OK; })                                                          \
  }                                                                                                                               \
  int orc_reduced_tmul_##SUFFIX(OrcQR* o, double* g, i64 ng, const double* w, i64 nw, const T* F) {                             \
    ORC_TRY({ reduced_tmul<T>(g, ng, w, nw, F, o->q); return ORC_OK; })                                                         \
  }                                                                                                                               \
  int orc_reduced_jacobian_dense_##SUFFIX(OrcQR* o, T* Jt, i64 nrows, i64 ncols, double* rt, i64 n_rt, const T* F, const double* Fr) { \
    ORC_TRY({ reduced_jacobian_dense<T>(Jt, nrows, ncols, rt, n_rt, F, Fr, o->q); return ORC_OK; })                              \
  }                                                                                                                               \
  int orc_reduced_jacobian_sparse_##SUFFIX(OrcQR* o, i64 nrows, i64 ncols, const i64* colptr0, const i64* rowval0, T* nzval,    \
                                           double* rt, i64 n_rt, const T* F, const double* Fr) {                                 \
    ORC_TRY({                                                                                                                     \
      IV cp(ncols + 1), rv(colptr0[ncols]);                                                                                       \
      for (i64 c = 0; c <= ncols; ++c) cp(c + 1) = colptr0[c] + 1;                                                                \
      for (i64 k = 0; k < colptr0[ncols]; ++k) rv(k + 1) = rowval0[k] + 1;                                                       \
      reduced_jacobian_sparse<T>(nrows, ncols, cp, rv, nzval, rt, n_rt, F, Fr, o->q);                                            \
      return ORC_OK;                                                                                                              \
    })                                                                                                                            \
  }                                                                                                                               \
  int orc_reduced_diagonal_blocks_##SUFFIX(OrcQR* o, T* D, const T* F) {                                                          \
    ORC_TRY({ reduced_diagonal_blocks<T>(D, F, o->q); return ORC_OK; })                                                          \
  }                                                                                                                               \
  int orc_factor_diagonal_blocks_##SUFFIX(T* D, const i64* dims, i64 nb) { return factor_diagonal_blocks<T>(D, dims, nb) ? ORC_OK : ORC_NOT_PD; } \
  void orc_solve_diagonal_blocks_##SUFFIX(double* y, const T* D, const i64* dims, i64 nb, const double* x) {                     \
    solve_diagonal_blocks<T>(y, D, dims, nb, x);                                                                                  \
  }

ORC_QR_TYPED(f64, double)
ORC_QR_TYPED(f32, float)

// the scalar-level build_r_to_s_map forms, 0-based in and out (0 -> -1 for an unmapped entry)
int orc_r_to_s_map_csc(i64 ncols, const i64* R_colptr, const i64* R_rowval, const i64* S_colptr, const i64* S_rowval, i64 S_ncols, i64* out) {
  ORC_TRY({
    IV rc(ncols + 1), rr(R_colptr[ncols]), sc(S_ncols + 1), sr(S_colptr[S_ncols]);
    for (i64 c = 0; c <= ncols; ++c) rc(c + 1) = R_colptr[c] + 1;
    for (i64 k = 0; k < R_colptr[ncols]; ++k) rr(k + 1) = R_rowval[k] + 1;
    for (i64 c = 0; c <= S_ncols; ++c) sc(c + 1) = S_colptr[c] + 1;
    for (i64 k = 0; k < S_colptr[S_ncols]; ++k) sr(k + 1) = S_rowval[k] + 1;
    IV m = r_to_s_map_csc(ncols, rc, rr, sc, sr);
    put(out, m.v, -1);
    return ORC_OK;
  })
}
int orc_r_to_s_map_blocks_csc(i64 nb, const i64* sizes, const i64* it_colptr, const i64* it_rowval, const i64* it_nzval, i64 data_len,
                              const i64* S_colptr, const i64* S_rowval, i64 S_ncols, const i64* boffsets_r, i64* out) {
  ORC_TRY({
    IV sz(nb), icp(nb + 1), irv(it_colptr[nb]), inz(it_colptr[nb]), sc(S_ncols + 1), sr(S_colptr[S_ncols]), bo(nb);
    for (i64 b = 0; b < nb; ++b) { sz(b + 1) = sizes[b]; bo(b + 1) = boffsets_r[b] + 1; }
    for (i64 b = 0; b <= nb; ++b) icp(b + 1) = it_colptr[b] + 1;
    for (i64 k = 0; k < it_colptr[nb]; ++k) { irv(k + 1) = it_rowval[k] + 1; inz(k + 1) = it_nzval[k] + 1; }
    for (i64 c = 0; c <= S_ncols; ++c) sc(c + 1) = S_colptr[c] + 1;
    for (i64 k = 0; k < S_colptr[S_ncols]; ++k) sr(k + 1) = S_rowval[k] + 1;
    IV m = r_to_s_map_blocks_csc(nb, sz, icp, irv, inz, data_len, sc, sr, bo);
    put(out, m.v, -1);
    return ORC_OK;
  })
}

int orc_reduced_residual(OrcQR* o, double* rt, i64 n_rt, const double* Fr) {
  ORC_TRY({ reduced_residual(rt, n_rt, Fr, o->q); return ORC_OK; })
}
// build_reduced_jacobian_pattern, 0-based: returns nnz; colptr (nr + 1) and rowval filled when not NULL
i64 orc_reduced_jacobian_pattern(OrcQR* o, i64* colptr, i64* rowval) {
  IV cp, rv;
  try { reduced_jacobian_pattern(o->q, cp, rv); } catch (const BlsError& e) { g_err = e.what(); return -1; }
  put(colptr, cp.v, -1);
  put(rowval, rv.v, -1);
  return rv.len();
}

int orc_pcg_solve_f64(OrcStructure* o, OrcPattern* p, const double* S, const double* g, double* x, double tol, i64 maxit, int nthreads,
                      i64* iters, double* rel) {
  ORC_TRY({ return pcg_solve<double>(o->st, p->P, S, g, x, tol, maxit, nthreads, iters, rel); })
}
int orc_pcg_solve_f32(OrcStructure* o, OrcPattern* p, const float* S, const double* g, double* x, double tol, i64 maxit, int nthreads,
                      i64* iters, double* rel) {
  ORC_TRY({ return pcg_solve<float>(o->st, p->P, S, g, x, tol, maxit, nthreads, iters, rel); })
}

// The closed-form inverse alone (tests of src/kernels.jl:14-67 and the generic path): d x d column-major H, damping
// scale (lambda = 1 folded into `damp`). Returns 1 on success.
int orc_inv_sym_block_f64(int d, const double* H, const double* damp, double* inv) {
  if (d == 1) return inv_sym_1<double>(H, damp, inv);
  if (d == 2) return inv_sym_2<double>(H, damp, inv);
  if (d == 3) return inv_sym_3<double>(H, damp, inv);
  return inv_sym_generic<double>(H, damp, inv, d, nullptr);
}
int orc_inv_sym_block_f32(int d, const float* H, const float* damp, float* inv) {
  if (d == 1) return inv_sym_1<float>(H, damp, inv);
  if (d == 2) return inv_sym_2<float>(H, damp, inv);
  if (d == 3) return inv_sym_3<float>(H, damp, inv);
  return inv_sym_generic<float>(H, damp, inv, d, nullptr);
}
int orc_inv_sym_block_generic_f64(int d, const double* H, const double* damp, double* inv) { return inv_sym_generic<double>(H, damp, inv, d, nullptr); }

int orc_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
