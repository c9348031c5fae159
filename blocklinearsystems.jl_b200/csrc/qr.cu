// QR elimination on sm_100a: reduce_qr!, the reduced normal equations J~'J~ and J~'r~, the diagonal blocks of J~'J~
// and the back-substitution x_e = U^-1 (q - B x_r).
//
// Reference: src/qr_reduction.jl (qr_table! :50-131, reduce_qr! :162-187, copy_table! :192-221, scale_table_columns!
// :225-255), src/qr_reduced.jl (qr_backsubstitute_group! :24-93, accumulate_qr_entry! :375-405, reduced_normal_* :409-480,
// reduced_diagonal_blocks! :484-512), layout src/schur_jacobian.jl:30-160.
//
// One warp per eliminated block's table: the table (M rows, C columns, column-major, contiguous in the raw storage) is
// copied into shared memory with coalesced loads, checked for non-finite entries, damped, and factored there: for each
// of the d_e eliminated columns the column norms, beta, tau and the reflector scaling are FP64 (warp reductions), and
// the reflector is applied with lanes owning columns, each lane walking its column down the rows (a table's row count
// M = m_e + d_e is odd whenever m_e is even, so the lanes' column strides hit distinct shared-memory banks). The
// residual column goes through the same reflectors in FP64 (SP-B6 of the reference). With FP32 storage (the mixed
// form) the table is FP32 and each reflector application is accumulated in FP64 and rounded once per entry.
#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>
#include <cmath>
#include <type_traits>

#include "common.cuh"

namespace bls {

constexpr long long QNONE = LLONG_MAX;
constexpr int QR_PAIR_CHUNK = 32;

struct QRPlan {
  bls_ctx* ctx = nullptr;
  int64_t nrblocks = 0, neblocks = 0, ntables = 0, nentries = 0, nr = 0, ne = 0, raw_len = 0, res_len = 0;
  int64_t max_cells = 0, max_rows = 0, nblocks = 0, nitems = 0, nnzS = 0;
  bool has_sparse = false;
  int max_dr = 0;
  // device: per table, per entry, per retained / eliminated block
  DevBuf t_rows, t_cols, t_top, t_raw, t_res, t_ptr, e_dims, boff_e;
  DevBuf u_ret, u_col, r_dims, boff_r, doff;
  // eliminated tables by shared-memory class (bytes of the staged table and residual, per element type)
  struct TableClass {
    DevBuf tables;
    int64_t n = 0, bytes_f64 = 0, bytes_f32 = 0;
  };
  TableClass classes[8];
  // J~'J~ work items (pairs of entries of one table, per S block)
  DevBuf pair_u1, pair_u2, item_block, item_start, item_info, blk_r1, blk_r2, blk_base_sparse, blk_stride, blk_base_dense;
  DevBuf r_ptr, r_entry, u_table;
  DevBuf status;
  long long* host_status = nullptr;
  int64_t launches = 0;
  ~QRPlan() { if (host_status) cudaFreeHost(host_status); }
};

static std::vector<int32_t> q32(const int64_t* a, int64_t n, const char* what) {
  std::vector<int32_t> v((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    if (a[i] < INT32_MIN || a[i] > INT32_MAX) throw Error(BLS_EUNSUPPORTED, std::string(what) + " exceeds the 32-bit index range of this build");
    v[i] = (int32_t)a[i];
  }
  return v;
}

// status: [0] lowest failing table, [1] lowest bad scaling_e entry
__global__ void k_qr_begin(long long* st) { st[0] = QNONE; st[1] = QNONE; }
__global__ void k_qr_check(const double* __restrict__ sc, int64_t n, long long* st) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = sc[i];
  if (!(isfinite(x) && x >= 0.0)) atomicMin(st + 1, (long long)i);
}

template <class T> __device__ __forceinline__ double eps_of();
template <> __device__ __forceinline__ double eps_of<double>() { return 2.220446049250313e-16; }
template <> __device__ __forceinline__ double eps_of<float>() { return 1.1920928955078125e-07; }

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Scale of table column j (the variable it belongs to): s over all variables [s_r; s_e]; 1 when s is null.
__device__ __forceinline__ double col_scale(const double* s, int j, int t, int ncols_f, int de, const int32_t* t_ptr, const int32_t* u_col,
                                            const int32_t* u_ret, const int32_t* boff_r, const int32_t* r_dims, const int32_t* boff_e, int nr) {
  if (!s) return 1.0;
  if (j >= ncols_f - de) return s[nr + boff_e[t] + (j - (ncols_f - de))];
  for (int u = t_ptr[t]; u < t_ptr[t + 1]; ++u) {
    const int c0 = u_col[u], r = u_ret[u];
    if (j >= c0 && j < c0 + r_dims[r]) return s[boff_r[r] + (j - c0)];
  }
  return 1.0;
}

// qr_table! for the listed eliminated tables, one warp per table; `shT` holds the table (M x C, column-major) and
// the FP64 residual (M). Tables are assigned by `tables[blockIdx.x * warps + warp]`.
template <class T>
__global__ void __launch_bounds__(32) k_qr_tables(int64_t ntab, const int32_t* __restrict__ tables, const int32_t* __restrict__ t_rows,
                                                  const int32_t* __restrict__ t_cols, const int64_t* __restrict__ t_raw,
                                                  const int64_t* __restrict__ t_res, const int32_t* __restrict__ t_ptr,
                                                  const int32_t* __restrict__ u_col, const int32_t* __restrict__ u_ret,
                                                  const int32_t* __restrict__ boff_r, const int32_t* __restrict__ r_dims,
                                                  const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boff_e, int nr,
                                                  const T* __restrict__ Rw, const double* __restrict__ Rr, const double* __restrict__ sc_e,
                                                  double lambda, const double* __restrict__ s, T* __restrict__ F, double* __restrict__ Fr,
                                                  long long* st) {
  extern __shared__ __align__(16) unsigned char qsm[];
  const int64_t wi = blockIdx.x;
  if (wi >= ntab) return;
  if (st[1] != QNONE) return;
  const int lane = threadIdx.x;
  const int t = tables[wi];
  const int M = t_rows[t], C = t_cols[t] - 1, de = e_dims[t], me = M - de, ce = C - de;
  const int64_t off = t_raw[t], rq = t_res[t];
  double* res = reinterpret_cast<double*>(qsm);
  T* A = reinterpret_cast<T*>(qsm + sizeof(double) * ((M + 1) & ~1));
  // copy in (coalesced: the table is contiguous), with the reference's non-finite test (x - x is NaN for Inf / NaN)
  bool bad = false;
  for (int i = lane; i < M * C; i += 32) {
    const int j = i / M;
    T x = Rw[off + i];
    bad |= isnan((double)(x - x));
    if (s) x = T((double)x * col_scale(s, j, t, C, de, t_ptr, u_col, u_ret, boff_r, r_dims, boff_e, nr));
    A[i] = x;
  }
  for (int i = lane; i < M; i += 32) {
    const double x = Rr[rq + i];
    bad |= isnan(x - x);
    res[i] = x;
  }
  bad = __any_sync(0xffffffffu, bad);
  if (bad) {
    if (lane == 0) atomicMin(st, (long long)t);
    return;
  }
  __syncwarp();
  // damping rows: zero, then sqrt(lambda * scaling_e) * s_e on their diagonal (formed in FP64)
  for (int i = lane; i < de * C; i += 32) {
    const int j = i / de, r = me + (i - j * de);
    A[j * M + r] = T(0);
  }
  for (int l = lane; l < de; l += 32) res[me + l] = 0.0;
  __syncwarp();
  for (int l = lane; l < de; l += 32) {
    const int so = boff_e[t];
    const double sv = s ? s[nr + so + l] : 1.0;
    A[(ce + l) * M + me + l] = T(sqrt(lambda * sc_e[so + l]) * sv);
  }
  __syncwarp();
  const double tol = (double)M * eps_of<T>();
  for (int k = 0; k < de; ++k) {
    T* col = A + (ce + k) * M;
    double s_top = 0.0, s_sub = 0.0;
    for (int i = lane; i < M; i += 32) {
      const double v = (double)col[i];
      if (i < k) s_top += v * v;
      else s_sub += v * v;
    }
    s_top = warp_sum(s_top);
    s_sub = warp_sum(s_sub);
    const double nrm = sqrt(s_sub), full = sqrt(s_top + s_sub);
    const double a = (double)col[k];
    const double beta = a >= 0.0 ? -nrm : nrm;
    if (!(isfinite(beta) && fabs(beta) > tol * full)) {
      if (lane == 0) atomicMin(st, (long long)t);
      return;
    }
    const double scale = 1.0 / (a - beta);
    const double tau = (beta - a) / beta;
    __syncwarp();
    for (int i = k + 1 + lane; i < M; i += 32) col[i] = T((double)col[i] * scale);
    __syncwarp();
    if (lane == 0) col[k] = T(beta);
    // apply I - tau v v' (v = [1; col[k+1:]]) to every column outside the eliminated columns ce..ce+k
    for (int j = lane; j < C; j += 32) {
      if (j >= ce && j <= ce + k) continue;
      T* y = A + j * M;
      double sj = (double)y[k];
      for (int i = k + 1; i < M; ++i) sj += (double)col[i] * (double)y[i];
      sj *= tau;
      y[k] = T((double)y[k] - sj);
      for (int i = k + 1; i < M; ++i) y[i] = T((double)y[i] - sj * (double)col[i]);
    }
    // and to the FP64 residual
    double sr = 0.0;
    for (int i = k + 1 + lane; i < M; i += 32) sr += (double)col[i] * res[i];
    sr = warp_sum(sr) + res[k];
    sr *= tau;
    __syncwarp();
    if (lane == 0) res[k] -= sr;
    for (int i = k + 1 + lane; i < M; i += 32) res[i] -= sr * (double)col[i];
    __syncwarp();
    for (int i = k + 1 + lane; i < M; i += 32) col[i] = T(0);
    __syncwarp();
  }
  for (int i = lane; i < M * C; i += 32) F[off + i] = A[i];
  for (int i = lane; i < M; i += 32) Fr[rq + i] = res[i];
}

// Free tables are copied (scaled when conditioned): copy_table! (src/qr_reduction.jl:183-185)
template <class T>
__global__ void k_qr_free(int64_t t0, int64_t nt, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_cols,
                          const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_res, const int32_t* __restrict__ t_ptr,
                          const int32_t* __restrict__ u_col, const int32_t* __restrict__ u_ret, const int32_t* __restrict__ boff_r,
                          const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_e, int nr, const T* __restrict__ Rw,
                          const double* __restrict__ Rr, const double* __restrict__ s, T* __restrict__ F, double* __restrict__ Fr,
                          const long long* st) {
  const int64_t t = t0 + blockIdx.x;
  if (t >= nt || st[0] != QNONE || st[1] != QNONE) return;
  const int M = t_rows[t], C = t_cols[t] - 1;
  const int64_t off = t_raw[t], rq = t_res[t];
  for (int i = threadIdx.x; i < M * C; i += blockDim.x) {
    T x = Rw[off + i];
    if (s) x = T((double)x * col_scale(s, i / M, (int)t, C, 0, t_ptr, u_col, u_ret, boff_r, r_dims, boff_e, nr));
    F[off + i] = x;
  }
  for (int i = threadIdx.x; i < M; i += blockDim.x) Fr[rq + i] = Rr[rq + i];
}

// J~'J~ and J~'r~ (accumulate_qr_entry!): six threads per work item (pairs (u1, u2) of one table with u1 <= u2, all of
// one S block), thread w owning column w of the block: sum over the pairs of the dots of the bottom n = M - top rows.
template <class T>
__global__ void __launch_bounds__(128) k_qr_pairs(int64_t nitems, const int32_t* __restrict__ item_block, const int32_t* __restrict__ item_start,
                                                  const int32_t* __restrict__ item_info, const int32_t* __restrict__ pair_u1,
                                                  const int32_t* __restrict__ pair_u2, const int32_t* __restrict__ blk_r1,
                                                  const int32_t* __restrict__ blk_r2, const int64_t* __restrict__ blk_base,
                                                  const int32_t* __restrict__ blk_stride, int64_t dense_nr, const int32_t* __restrict__ u_table,
                                                  const int32_t* __restrict__ u_col, const int32_t* __restrict__ t_rows,
                                                  const int32_t* __restrict__ t_top, const int64_t* __restrict__ t_raw,
                                                  const int64_t* __restrict__ t_res, const int32_t* __restrict__ r_dims,
                                                  const int32_t* __restrict__ boff_r, const T* __restrict__ F, const double* __restrict__ Fr,
                                                  T* __restrict__ S, double* __restrict__ g) {
  const int lane = threadIdx.x & 31;
  if (lane >= 30) return;
  const int64_t it = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 5 + lane / 6;
  if (it >= nitems) return;
  const int k = item_block[it], pb = item_start[it], info = item_info[it];
  const int pe = pb + (info & 0xffff);
  const bool solo = (info >> 16) != 0;
  const int r1 = blk_r1[k], r2 = blk_r2[k];
  const bool diag = r1 == r2;
  const int d1 = r_dims[r1], d2 = r_dims[r2];
  const int64_t stride = blk_stride ? (int64_t)blk_stride[k] : dense_nr;
  for (int w = lane % 6; w < d2; w += 6) {
    double acc[16];
#pragma unroll
    for (int a = 0; a < 16; ++a) acc[a] = 0.0;
    double gacc = 0.0;
    for (int p = pb; p < pe; ++p) {
      const int u1 = pair_u1[p], u2 = pair_u2[p], t = u_table[u2];
      const int M = t_rows[t], top = t_top[t], n = M - top;
      const T* base = F + t_raw[t] + top;
      const T* yw = base + (int64_t)(u_col[u2] + w) * M;
      const T* x0 = base + (int64_t)u_col[u1] * M;
      const double* rr = Fr + t_res[t] + top;
      for (int i = 0; i < n; ++i) {
        const double yv = (double)yw[i];
#pragma unroll
        for (int a = 0; a < 16; ++a)
          if (a < d1) acc[a] += (double)x0[(int64_t)a * M + i] * yv;
        if (diag) gacc += yv * rr[i];
      }
    }
    T* colp = S + blk_base[k] + w * stride;
#pragma unroll
    for (int a = 0; a < 16; ++a) {
      if (a >= d1 || (diag && a > w)) continue;
      if (solo) colp[a] = T((double)colp[a] + acc[a]);
      else atomicAdd(colp + a, T(acc[a]));
    }
    if (diag) {
      if (solo) g[boff_r[r2] + w] += gacc;
      else atomicAdd(g + boff_r[r2] + w, gacc);
    }
  }
}

// reduced_diagonal_blocks!: thread (r, w) sums column w of J~_u' J~_u over the entries u of retained block r
template <class T>
__global__ void k_qr_diag(int64_t nrb, const int32_t* __restrict__ r_ptr, const int32_t* __restrict__ r_entry, const int32_t* __restrict__ u_table,
                          const int32_t* __restrict__ u_col, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_top,
                          const int64_t* __restrict__ t_raw, const int32_t* __restrict__ r_dims, const int64_t* __restrict__ doff,
                          const T* __restrict__ F, T* __restrict__ D) {
  const int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t r = id >> 4;
  const int w = (int)(id & 15);
  if (r >= nrb) return;
  const int dr = r_dims[r];
  if (w >= dr) return;
  double acc[16];
#pragma unroll
  for (int a = 0; a < 16; ++a) acc[a] = 0.0;
  for (int q = r_ptr[r]; q < r_ptr[r + 1]; ++q) {
    const int u = r_entry[q], t = u_table[u];
    const int M = t_rows[t], top = t_top[t];
    const T* base = F + t_raw[t] + top + (int64_t)u_col[u] * M;
    for (int i = 0; i < M - top; ++i) {
      const double yv = (double)base[(int64_t)w * M + i];
#pragma unroll
      for (int a = 0; a < 16; ++a)
        if (a < dr) acc[a] += (double)base[(int64_t)a * M + i] * yv;
    }
  }
#pragma unroll
  for (int a = 0; a < 16; ++a)
    if (a < dr) D[doff[r] + (int64_t)w * dr + a] = T(acc[a]);
}

// qr_backsubstitute_group! (src/qr_reduced.jl:24-93): thread per eliminated table, FP64
template <class T>
__global__ void k_qr_backsub(int64_t ne_tab, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_cols,
                             const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_res, const int32_t* __restrict__ t_ptr,
                             const int32_t* __restrict__ u_col, const int32_t* __restrict__ u_ret, const int32_t* __restrict__ r_dims,
                             const int32_t* __restrict__ boff_r, const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boff_e,
                             const T* __restrict__ F, const double* __restrict__ Fr, const double* __restrict__ x_r, double* __restrict__ x_e) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne_tab) return;
  const int M = t_rows[e], C = t_cols[e], de = e_dims[e], ce = C - de - 1;
  const int64_t off = t_raw[e];
  // t = q - B x_r accumulated in x_e's own entries, then U x_e = t solved in place (the same operations in the same order)
  double* xe = x_e + boff_e[e];
  for (int i = 0; i < de; ++i) xe[i] = Fr[t_res[e] + i];
  for (int u = t_ptr[e]; u < t_ptr[e + 1]; ++u) {
    const int r = u_ret[u], ro = boff_r[r];
    const T* cb = F + off + (int64_t)u_col[u] * M;
    for (int j = 0; j < r_dims[r]; ++j) {
      const double xj = x_r[ro + j];
      for (int i = 0; i < de; ++i) xe[i] -= (double)cb[(int64_t)j * M + i] * xj;
    }
  }
  for (int i = de - 1; i >= 0; --i) {
    double acc = xe[i];
    for (int j = i + 1; j < de; ++j) acc -= (double)F[off + (int64_t)(ce + j) * M + i] * xe[j];
    xe[i] = acc / (double)F[off + (int64_t)(ce + i) * M + i];
  }
}

template <class T>
__global__ void k_fill_t(T* __restrict__ p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = T(0);
}

// ------------------------------------------------------------------------------------------------------------------
// Plan
// ------------------------------------------------------------------------------------------------------------------
static QRPlan* qr_plan_create(bls_ctx* ctx, const bls_qr_plan_desc* d) {
  if (!d || d->nrblocks < 1 || d->neblocks < 1 || d->ntables < d->neblocks) throw Error(BLS_EINVAL, "a QR plan needs retained blocks, eliminated blocks and their tables");
  std::unique_ptr<QRPlan> P(new QRPlan());
  P->ctx = ctx;
  cudaStream_t s = ctx->stream;
  const int64_t nrb = d->nrblocks, neb = d->neblocks, nt = d->ntables;
  P->nrblocks = nrb; P->neblocks = neb; P->ntables = nt;
  const int64_t nent = d->table_ptr[nt];
  P->nentries = nent;
  std::vector<int64_t> boff_r(nrb), boff_e(neb), doff(nrb + 1, 0);
  int64_t nr = 0, ne = 0;
  for (int64_t r = 0; r < nrb; ++r) {
    if (d->r_dims[r] < 1 || d->r_dims[r] > 16) throw Error(BLS_EUNSUPPORTED, "retained block sizes above 16 are not supported on the device");
    boff_r[r] = nr; nr += d->r_dims[r];
    doff[r + 1] = doff[r] + d->r_dims[r] * d->r_dims[r];
    P->max_dr = std::max<int>(P->max_dr, (int)d->r_dims[r]);
  }
  for (int64_t e = 0; e < neb; ++e) {
    if (d->e_dims[e] < 1) throw Error(BLS_EINVAL, "eliminated block sizes must be positive");
    boff_e[e] = ne; ne += d->e_dims[e];
  }
  P->nr = nr; P->ne = ne;
  // tables: consistency checks that keep every device access inside the caller's buffers
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t M = d->table_nrows[t], C = d->table_ncols[t] - 1;
    const int64_t de = t < neb ? d->e_dims[t] : 0;
    if (M < 1 || C < de || d->table_top[t] != de || d->raw_offsets[t + 1] - d->raw_offsets[t] != M * C ||
        d->residual_offsets[t + 1] - d->residual_offsets[t] != M)
      throw Error(BLS_EINVAL, "table " + std::to_string(t + 1) + " has an inconsistent layout");
    int64_t col = 0;
    for (int64_t u = d->table_ptr[t]; u < d->table_ptr[t + 1]; ++u) {
      const int64_t r = d->entry_retained[u];
      if (r < 0 || r >= nrb || d->entry_col[u] != col) throw Error(BLS_EINVAL, "table " + std::to_string(t + 1) + " has malformed entries");
      col += d->r_dims[r];
    }
    if (col + de != C) throw Error(BLS_EINVAL, "table " + std::to_string(t + 1) + ": entries do not fill its columns");
    P->max_rows = std::max(P->max_rows, M);
  }
  P->raw_len = d->raw_offsets[nt];
  P->res_len = d->residual_offsets[nt];
  // shared-memory classes of the eliminated tables by their FP64 footprint (residual rounded to an even row count, then
  // the M x C table): <= 2, 4, 8, 16, 32, 64, 128, 224 KB
  std::vector<int32_t> cls_tables[8];
  for (int64_t t = 0; t < neb; ++t) {
    const int64_t M = d->table_nrows[t], C = d->table_ncols[t] - 1;
    const int64_t b64 = 8 * ((M + 1) & ~1) + 8 * M * C, b32 = 8 * ((M + 1) & ~1) + 4 * M * C;
    int c = 0;
    while (c < 7 && b64 > (int64_t(2048) << c)) ++c;
    if (b64 > 224 * 1024) throw Error(BLS_EUNSUPPORTED, "table " + std::to_string(t + 1) + " exceeds the shared-memory capacity of this build");
    cls_tables[c].push_back((int32_t)t);
    P->classes[c].bytes_f64 = std::max(P->classes[c].bytes_f64, b64);
    P->classes[c].bytes_f32 = std::max(P->classes[c].bytes_f32, b32);
  }
  // per entry: table; per retained block: its entries (ascending)
  std::vector<int32_t> u_table(nent), rptr(nrb + 1, 0), rentry(nent);
  for (int64_t t = 0; t < nt; ++t)
    for (int64_t u = d->table_ptr[t]; u < d->table_ptr[t + 1]; ++u) { u_table[u] = (int32_t)t; rptr[d->entry_retained[u] + 1] += 1; }
  for (int64_t r = 0; r < nrb; ++r) rptr[r + 1] += rptr[r];
  {
    std::vector<int32_t> fill(rptr.begin(), rptr.end() - 1);
    for (int64_t u = 0; u < nent; ++u) rentry[fill[d->entry_retained[u]]++] = (int32_t)u;
  }
  // J~'J~ blocks: the given pattern, or the tables' own block pattern
  std::vector<int64_t> bcolptr, browval, brow_off, col_h, Scolptr;
  P->has_sparse = d->block_colptr != nullptr;
  if (P->has_sparse) {
    bcolptr.assign(d->block_colptr, d->block_colptr + nrb + 1);
    browval.assign(d->block_rowval, d->block_rowval + bcolptr[nrb]);
    brow_off.assign(d->block_row_offsets, d->block_row_offsets + bcolptr[nrb]);
    col_h.assign(d->col_heights, d->col_heights + nrb);
    Scolptr.assign(d->S_colptr, d->S_colptr + nr + 1);
    P->nnzS = Scolptr[nr];
    for (int64_t r2 = 0; r2 < nrb; ++r2) {
      for (int64_t w = 0; w < d->r_dims[r2]; ++w)
        if (Scolptr[boff_r[r2] + w + 1] - Scolptr[boff_r[r2] + w] != col_h[r2]) throw Error(BLS_EINVAL, "S_colptr does not match col_heights");
      for (int64_t k = bcolptr[r2]; k < bcolptr[r2 + 1]; ++k)
        if (browval[k] < 0 || browval[k] > r2 || brow_off[k] < 0 || brow_off[k] + d->r_dims[browval[k]] > col_h[r2])
          throw Error(BLS_EINVAL, "malformed block pattern");
    }
  } else {
    std::vector<std::vector<int64_t>> cols(nrb);
    for (int64_t t = 0; t < nt; ++t)
      for (int64_t u2 = d->table_ptr[t]; u2 < d->table_ptr[t + 1]; ++u2)
        for (int64_t u1 = d->table_ptr[t]; u1 <= u2; ++u1) cols[d->entry_retained[u2]].push_back(d->entry_retained[u1]);
    bcolptr.assign(nrb + 1, 0);
    for (int64_t r = 0; r < nrb; ++r) {
      auto& v = cols[r];
      v.push_back(r);
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      bcolptr[r + 1] = bcolptr[r] + (int64_t)v.size();
      int64_t h = 0;
      for (int64_t x : v) { browval.push_back(x); brow_off.push_back(h); h += d->r_dims[x]; }
      col_h.push_back(h);
    }
  }
  const int64_t nb = bcolptr[nrb];
  P->nblocks = nb;
  std::vector<int32_t> b_r1(nb), b_r2(nb), b_stride(nb);
  std::vector<int64_t> b_base(nb, 0), b_base_dense(nb);
  for (int64_t r2 = 0; r2 < nrb; ++r2)
    for (int64_t k = bcolptr[r2]; k < bcolptr[r2 + 1]; ++k) {
      b_r1[k] = (int32_t)browval[k];
      b_r2[k] = (int32_t)r2;
      b_stride[k] = (int32_t)col_h[r2];
      if (P->has_sparse) b_base[k] = Scolptr[boff_r[r2]] + brow_off[k];
      b_base_dense[k] = boff_r[browval[k]] + boff_r[r2] * nr;
    }
  // pairs (u1, u2), u1 <= u2 of one table, per block (r1, r2), in ascending table order
  std::vector<int32_t> pu1, pu2, itb, its, iti;
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    const int64_t kb = bcolptr[r2], ke = bcolptr[r2 + 1];
    std::vector<std::vector<std::pair<int32_t, int32_t>>> per(ke - kb);
    for (int32_t q = rptr[r2]; q < rptr[r2 + 1]; ++q) {
      const int32_t u2 = rentry[q];
      const int64_t t = u_table[u2];
      for (int64_t u1 = d->table_ptr[t]; u1 <= u2; ++u1) {
        const int64_t r1 = d->entry_retained[u1];
        const int64_t* f = std::lower_bound(browval.data() + kb, browval.data() + ke, r1);
        if (f == browval.data() + ke || *f != r1) throw Error(BLS_EPATTERN, "The sparse pattern has no block (" + std::to_string(r1 + 1) + ", " + std::to_string(r2 + 1) + ")");
        per[f - (browval.data() + kb)].push_back({(int32_t)u1, u2});
      }
    }
    for (int64_t sl = 0; sl < ke - kb; ++sl) {
      const auto& v = per[sl];
      const int nch = ((int)v.size() + QR_PAIR_CHUNK - 1) / QR_PAIR_CHUNK;
      for (size_t x = 0; x < v.size(); x += QR_PAIR_CHUNK) {
        itb.push_back((int32_t)(kb + sl));
        its.push_back((int32_t)pu1.size() + 0);
        const int cnt = (int)std::min<size_t>(QR_PAIR_CHUNK, v.size() - x);
        iti.push_back(cnt | ((nch == 1 ? 1 : 0) << 16));
        for (int y = 0; y < cnt; ++y) { pu1.push_back(v[x + y].first); pu2.push_back(v[x + y].second); }
      }
    }
  }
  P->nitems = (int64_t)itb.size();
  std::vector<int32_t> t_rows = q32(d->table_nrows, nt, "table_nrows"), t_cols = q32(d->table_ncols, nt, "table_ncols"),
                       t_top = q32(d->table_top, nt, "table_top"), t_ptr = q32(d->table_ptr, nt + 1, "table_ptr");
  upload(P->t_rows, t_rows, s); upload(P->t_cols, t_cols, s); upload(P->t_top, t_top, s); upload(P->t_ptr, t_ptr, s);
  upload(P->t_raw, std::vector<int64_t>(d->raw_offsets, d->raw_offsets + nt + 1), s);
  upload(P->t_res, std::vector<int64_t>(d->residual_offsets, d->residual_offsets + nt + 1), s);
  upload(P->e_dims, q32(d->e_dims, neb, "e_dims"), s);
  upload(P->boff_e, q32(boff_e.data(), neb, "boffsets_e"), s);
  upload(P->u_ret, q32(d->entry_retained, nent, "entry_retained"), s);
  upload(P->u_col, q32(d->entry_col, nent, "entry_col"), s);
  upload(P->r_dims, q32(d->r_dims, nrb, "r_dims"), s);
  upload(P->boff_r, q32(boff_r.data(), nrb, "boffsets_r"), s);
  upload(P->doff, doff, s);
  for (int c = 0; c < 8; ++c) {
    P->classes[c].n = (int64_t)cls_tables[c].size();
    upload(P->classes[c].tables, cls_tables[c], s);
  }
  upload(P->u_table, u_table, s);
  upload(P->r_ptr, rptr, s);
  upload(P->r_entry, rentry, s);
  upload(P->pair_u1, pu1, s); upload(P->pair_u2, pu2, s);
  upload(P->item_block, itb, s); upload(P->item_start, its, s); upload(P->item_info, iti, s);
  upload(P->blk_r1, b_r1, s); upload(P->blk_r2, b_r2, s); upload(P->blk_stride, b_stride, s);
  upload(P->blk_base_sparse, b_base, s); upload(P->blk_base_dense, b_base_dense, s);
  P->status.alloc(4 * sizeof(long long));
  long long init[4] = {QNONE, QNONE, QNONE, QNONE};
  BLS_CUDA(cudaMemcpyAsync(P->status.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
  BLS_CUDA(cudaMallocHost(&P->host_status, 4 * sizeof(long long)));
  BLS_CUDA(cudaStreamSynchronize(s));
  return P.release();
}

template <class T>
static int reduce_qr(QRPlan* P, T* F, double* Fr, const T* Rw, const double* Rr, const double* sc_e, double lambda, const double* sv,
                     int64_t* failed_block) {
  if (!(std::isfinite(lambda) && lambda >= 0)) throw Error(BLS_EINVAL, "lambda must be finite and non-negative, got " + std::to_string(lambda));
  cudaStream_t s = P->ctx->stream;
  long long* st = P->status.as<long long>();
  k_qr_begin<<<1, 1, 0, s>>>(st);
  k_qr_check<<<grid_for(P->ne, 256), 256, 0, s>>>(sc_e, P->ne, st);
  P->launches += 2;
  for (int c = 0; c < 8; ++c) {
    const auto& k = P->classes[c];
    if (k.n == 0) continue;
    const size_t smem = (size_t)(std::is_same<T, double>::value ? k.bytes_f64 : k.bytes_f32);
    if (smem > 48 * 1024) BLS_CUDA(cudaFuncSetAttribute(k_qr_tables<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_qr_tables<T><<<(unsigned)k.n, 32, smem, s>>>(k.n, k.tables.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(),
                                                   P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(),
                                                   P->u_ret.as<int32_t>(), P->boff_r.as<int32_t>(), P->r_dims.as<int32_t>(),
                                                   P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(), (int)P->nr, Rw, Rr, sc_e, lambda, sv, F,
                                                   Fr, st);
    P->launches += 1;
  }
  if (P->ntables > P->neblocks) {
    k_qr_free<T><<<(unsigned)(P->ntables - P->neblocks), 128, 0, s>>>(P->neblocks, P->ntables, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(),
                                                                       P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(),
                                                                       P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(), P->boff_r.as<int32_t>(),
                                                                       P->r_dims.as<int32_t>(), P->boff_e.as<int32_t>(), (int)P->nr, Rw, Rr, sv,
                                                                       F, Fr, st);
    P->launches += 1;
  }
  BLS_CUDA(cudaGetLastError());
  if (!failed_block) return BLS_OK;
  BLS_CUDA(cudaMemcpyAsync(P->host_status, st, 2 * sizeof(long long), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  *failed_block = 0;
  if (P->host_status[1] != QNONE) {
    set_error("scaling_e must be finite and non-negative, but entry " + std::to_string(P->host_status[1] + 1) + " is not");
    return BLS_EINVAL;
  }
  if (P->host_status[0] != QNONE) {
    *failed_block = P->host_status[0] + 1;
    return BLS_NOT_PD;
  }
  return BLS_OK;
}

template <class T>
static void normal(QRPlan* P, T* S, bool dense, double* g, const T* F, const double* Fr) {
  if (!dense && !P->has_sparse) throw Error(BLS_EINVAL, "the QR plan was created without a sparse pattern");
  cudaStream_t s = P->ctx->stream;
  const int64_t nS = dense ? P->nr * P->nr : P->nnzS;
  k_fill_t<T><<<(unsigned)std::min<int64_t>(grid_for(nS, 256), 148 * 8), 256, 0, s>>>(S, nS);
  k_fill_t<double><<<grid_for(P->nr, 256), 256, 0, s>>>(g, P->nr);
  if (P->nitems > 0)
    k_qr_pairs<T><<<grid_for((P->nitems + 4) / 5 * 32, 128), 128, 0, s>>>(
        P->nitems, P->item_block.as<int32_t>(), P->item_start.as<int32_t>(), P->item_info.as<int32_t>(), P->pair_u1.as<int32_t>(),
        P->pair_u2.as<int32_t>(), P->blk_r1.as<int32_t>(), P->blk_r2.as<int32_t>(),
        dense ? P->blk_base_dense.as<int64_t>() : P->blk_base_sparse.as<int64_t>(), dense ? nullptr : P->blk_stride.as<int32_t>(), P->nr,
        P->u_table.as<int32_t>(), P->u_col.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(),
        P->t_res.as<int64_t>(), P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), F, Fr, S, g);
  P->launches += 3;
  BLS_CUDA(cudaGetLastError());
}

}  // namespace bls

struct bls_qr_plan : bls::QRPlan {};
using namespace bls;

#define QR_GUARD(...)                         \
  try {                                       \
    __VA_ARGS__                               \
  } catch (const bls::Error& e) {             \
    bls::set_error(e.what());                 \
    return e.code;                            \
  } catch (const std::bad_alloc&) {           \
    bls::set_error("out of host memory");     \
    return BLS_ENOMEM;                        \
  }

extern "C" {

int bls_qr_plan_create(bls_ctx* ctx, const bls_qr_plan_desc* desc, bls_qr_plan** out) {
  QR_GUARD({
    if (!ctx || !out) throw Error(BLS_EINVAL, "null argument");
    BLS_CUDA(cudaSetDevice(ctx->device));
    *out = static_cast<bls_qr_plan*>(qr_plan_create(ctx, desc));
    return BLS_OK;
  })
}

int bls_qr_plan_destroy(bls_qr_plan* plan) {
  if (plan) {
    cudaStreamSynchronize(plan->ctx->stream);
    delete static_cast<QRPlan*>(plan);
  }
  return BLS_OK;
}

int bls_reduce_qr(bls_qr_plan* P, int dtype, void* F, double* Fr, const void* Rw, const double* Rr, const double* scaling_e, double lambda,
                  const double* s, int64_t* failed_block) {
  QR_GUARD({
    if (dtype == BLS_F64) return reduce_qr<double>(P, (double*)F, Fr, (const double*)Rw, Rr, scaling_e, lambda, s, failed_block);
    if (dtype == BLS_F32) return reduce_qr<float>(P, (float*)F, Fr, (const float*)Rw, Rr, scaling_e, lambda, s, failed_block);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_qr_backsubstitute(bls_qr_plan* P, int dtype, double* x_e, const double* x_r, const void* F, const double* Fr) {
  QR_GUARD({
    cudaStream_t s = P->ctx->stream;
    if (dtype == BLS_F64)
      k_qr_backsub<double><<<grid_for(P->neblocks, 128), 128, 0, s>>>(P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(),
                                                                     P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(),
                                                                     P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(), P->r_dims.as<int32_t>(),
                                                                     P->boff_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(),
                                                                     (const double*)F, Fr, x_r, x_e);
    else if (dtype == BLS_F32)
      k_qr_backsub<float><<<grid_for(P->neblocks, 128), 128, 0, s>>>(P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(),
                                                                    P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(),
                                                                    P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(), P->r_dims.as<int32_t>(),
                                                                    P->boff_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(),
                                                                    (const float*)F, Fr, x_r, x_e);
    else throw Error(BLS_EINVAL, "unknown dtype");
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_reduced_normal_sparse(bls_qr_plan* P, int dtype, void* S, double* g, const void* F, const double* Fr) {
  QR_GUARD({
    if (dtype == BLS_F64) normal<double>(P, (double*)S, false, g, (const double*)F, Fr);
    else if (dtype == BLS_F32) normal<float>(P, (float*)S, false, g, (const float*)F, Fr);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_reduced_normal_dense(bls_qr_plan* P, int dtype, void* S, double* g, const void* F, const double* Fr) {
  QR_GUARD({
    if (dtype == BLS_F64) normal<double>(P, (double*)S, true, g, (const double*)F, Fr);
    else if (dtype == BLS_F32) normal<float>(P, (float*)S, true, g, (const float*)F, Fr);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_reduced_diagonal_blocks(bls_qr_plan* P, int dtype, void* D, const void* F) {
  QR_GUARD({
    cudaStream_t s = P->ctx->stream;
    const unsigned grid = (unsigned)grid_for(P->nrblocks * 16, 128);
    if (dtype == BLS_F64)
      k_qr_diag<double><<<grid, 128, 0, s>>>(P->nrblocks, P->r_ptr.as<int32_t>(), P->r_entry.as<int32_t>(), P->u_table.as<int32_t>(),
                                             P->u_col.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(),
                                             P->r_dims.as<int32_t>(), P->doff.as<int64_t>(), (const double*)F, (double*)D);
    else if (dtype == BLS_F32)
      k_qr_diag<float><<<grid, 128, 0, s>>>(P->nrblocks, P->r_ptr.as<int32_t>(), P->r_entry.as<int32_t>(), P->u_table.as<int32_t>(),
                                            P->u_col.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(),
                                            P->r_dims.as<int32_t>(), P->doff.as<int64_t>(), (const float*)F, (float*)D);
    else throw Error(BLS_EINVAL, "unknown dtype");
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

}  // extern "C"
