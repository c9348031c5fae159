// QR elimination on sm_100a: reduce_qr!, the reduced normal equations J~'J~ and J~'r~, the diagonal blocks of J~'J~
// and the back-substitution x_e = U^-1 (q - B x_r).
//
// Reference: src/qr_reduction.jl (qr_table! :50-131, reduce_qr! :162-187, copy_table! :192-221, scale_table_columns!
// :225-255), src/qr_reduced.jl (qr_backsubstitute_group! :24-93, accumulate_qr_entry! :375-405, reduced_normal_* :409-480,
// reduced_diagonal_blocks! :484-512), layout src/schur_jacobian.jl:30-160.
//
// A group of 8, 16 or 32 lanes per eliminated block's table: the table (M rows, C columns, column-major, contiguous in
// the raw storage) is copied into shared memory by a bulk copy, checked for non-finite entries, damped, and factored
// there. The d_e eliminated columns come first: for each, the column norms, beta, tau and the reflector scaling are FP64
// (group reductions), and the reflector is applied to the later eliminated columns. For d_e <= 4 the d_e reflectors then
// reach every retained column at once in compact form (y - V s with a = V'y and a d_e x d_e triangular recurrence for
// s), a lane per column reading its column twice; larger blocks take the reflectors one at a time, lanes owning
// columns. The residual column goes through the same reflectors in FP64 (SP-B6 of the reference). With FP32 storage
// (the mixed form) the table and its column updates are FP32, the norms, tau and s FP64. The factored table goes back by
// a bulk copy of its 16-byte-aligned interior.
//
// J~'J~, J~'r~ and the diagonal blocks come from one warp per table as well: the table's bottom rows (J~ of its
// retained columns) and residual rows are staged in shared memory, every pair of the table's entries (u1 <= u2)
// gives one d_r x d_r block, one lane per block column holding its FP64 dot products in registers, and the block is
// added into S with one atomic add per entry (a table contributes to each S block at most once). Tables are grouped into shared-memory classes;
// each class is one launch whose CTA size packs an SM's shared memory best, and the classes of one call run
// concurrently on the plan's side streams.
#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <cmath>
#include <type_traits>

#include "bulk.cuh"
#include "common.cuh"

namespace bls {

constexpr long long QNONE = LLONG_MAX;
constexpr int QR_MAX_WARPS = 4;
constexpr int64_t QR_SMEM_LIMIT = 220 * 1024;

struct QRPlan {
  bls_ctx* ctx = nullptr;
  int64_t nrblocks = 0, neblocks = 0, ntables = 0, nentries = 0, nr = 0, ne = 0, raw_len = 0, res_len = 0;
  int64_t max_rows = 0, nblocks = 0, nnzS = 0, ndiag = 0;
  bool has_sparse = false;
  bool all6 = true;   // every retained block has 6 columns (the Gram kernel's 6 x 6 form only)
  bool bulk = true;   // stage tables with bulk copies (false: element copies; bls_qr_plan_set_staging)
  int max_dr = 0;
  int max_de = 0;
  // device: per table, per entry, per retained / eliminated block
  DevBuf t_rows, t_cols, t_top, t_raw, t_res, t_ptr, e_dims, boff_e;
  DevBuf u_ret, u_col, r_dims, boff_r, doff;
  // tables by shared-memory class (bytes of what one warp stages, per element type): the eliminated tables for the
  // factorisation, every table for the Gram kernel
  struct TableClass {
    DevBuf tables;
    int64_t n = 0, bytes_f64 = 0, bytes_f32 = 0;
    int64_t maxc = 0;   // the widest table's column count (the factorisation's lanes per table follow it)
  };
  TableClass classes[8], gram_classes[8];
  // per table, per pair (u1 <= u2) of its entries in the order u2 outer, u1 inner: the S block it adds to
  DevBuf tp_ptr, tp_blk, blk_base_sparse, blk_stride, blk_base_dense;
  // the SchurBlockHessian layout of the same structure (assembly): E offset per eliminated block, C offset per entry of
  // an eliminated table (its coupling), and the lengths
  DevBuf t_eoff, u_coff;
  int64_t E_len = 0, C_len = 0;
  // per retained block its entries in ascending order (the structure's retained_ptr / retained_entry), per entry its table
  DevBuf q_rptr, q_rent, u_tab;
  DevBuf q_total;   // one FP64 accumulator (jtj_quadform)
  // the reduced problem (reduced_residual!, reduced_jacobian!): per table its first reduced row (t_red, nt + 1), the
  // CSC column pointers of J~ (build_reduced_jacobian_pattern, nr + 1, also kept on the host to check a caller's
  // pattern) and per entry the position of its run within each column of its retained block
  DevBuf t_red, jt_colptr, u_runpos;
  int64_t red_nrows = 0;
  std::vector<int64_t> h_red, h_jt_colptr;
  std::vector<int32_t> h_rptr, h_rent_tab;   // per retained block, the tables of its entries in ascending entry order
  std::vector<int64_t> h_boff_r, h_rdims;
  // LSMR on the reduced problem (allocated at its first call): the augmented vector u (reduced_nrows + nr), v, h, hbar and two scratch vectors (nr), sqrt(lambda s_r), the per-(entry, column pair)
  // products of the diagonal blocks, their FP64 Cholesky factors, the norm accumulators and the factorisation's flag
  // reduced_tmul!'s per-(entry, column) dot products (allocated at its first call), rdmax = the largest retained block
  DevBuf tm_part, red_tab, u_meta;
  int rdmax = 0;
  DevBuf ls_u, ls_v, ls_h, ls_hbar, ls_t, ls_w, ls_sqd, ls_part, ls_L, ls_acc, ls_flag;
  double* ls_host = nullptr;
  DevBuf status;
  long long* host_status = nullptr;
  int64_t launches = 0;
  // side streams of the per-class launches (factorisation and Gram kernels; created at the first use): the classes
  // run concurrently, so that one class's last wave overlaps the others' and small classes fill the SMs beside large
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[3] = {nullptr, nullptr, nullptr};
  ~QRPlan() {
    if (host_status) cudaFreeHost(host_status);
    if (ls_host) cudaFreeHost(ls_host);
    for (int i = 0; i < 3; ++i) {
      if (side[i]) cudaStreamDestroy(side[i]);
      if (ev_join[i]) cudaEventDestroy(ev_join[i]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
  }
};

static std::vector<int32_t> q32(const int64_t* a, int64_t n, const char* what) {
  std::vector<int32_t> v((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    if (a[i] < INT32_MIN || a[i] > INT32_MAX) throw Error(BLS_EUNSUPPORTED, std::string(what) + " exceeds the 32-bit index range of this build");
    v[i] = (int32_t)a[i];
  }
  return v;
}

// Warps per CTA for a per-warp shared-memory footprint: up to QR_MAX_WARPS within the shared-memory limit.
static int warps_per_cta(int64_t warp_bytes) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(QR_MAX_WARPS, QR_SMEM_LIMIT / std::max<int64_t>(warp_bytes, 1)));
}
// Tables per CTA of the factorisation with G lanes per table: whole warps (32 / G tables each), up to QR_MAX_WARPS
// within the shared-memory limit; 0 when not even one warp's tables fit.
// The warps of `kernel` that an SM's 64 K registers hold (cached per kernel).
static int warp_cap(const void* kernel) {
  static std::mutex mu;
  static std::map<const void*, int> cap;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cap.find(kernel);
  if (it != cap.end()) return it->second;
  cudaFuncAttributes a;
  BLS_CUDA(cudaFuncGetAttributes(&a, kernel));
  const int regs = (std::max(a.numRegs, 1) + 7) / 8 * 8;
  return cap[kernel] = std::max(1, std::min(64, 65536 / (regs * 32)));
}

// Of the CTA sizes that fit, the one that keeps the most warps resident on an SM (228 KB of shared memory, 1 KB of it
// reserved per CTA; at most 32 CTAs and `max_warps` warps by registers), the larger one on a tie: a large table class
// in four-warp CTAs would leave a quarter of an SM's shared memory unused.
static int tables_per_cta(int64_t table_bytes, int G, int max_warps) {
  const int64_t per_warp = 32 / G, warp_bytes = per_warp * std::max<int64_t>(table_bytes, 1);
  int64_t best_w = 0, best = 0;
  for (int64_t w = 1; w <= QR_MAX_WARPS && w * warp_bytes <= QR_SMEM_LIMIT; ++w) {
    const int64_t ctas = std::min<int64_t>(32, (228 * 1024) / (w * warp_bytes + 1024));
    const int64_t warps = std::min<int64_t>(max_warps, ctas * w);
    if (warps >= best) {
      best = warps;
      best_w = w;
    }
  }
  return (int)(best_w * per_warp);
}

static void set_smem(const void* kernel, size_t bytes) {
  if (bytes > 48 * 1024) BLS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// Fork the plan's side streams off s (they wait for all work issued on s so far); class q of a run of per-class
// launches goes to class_stream(P, s, q), and join_sides makes s wait for the side streams' work.
static void fork_sides(QRPlan* P, cudaStream_t s) {
  if (!P->ev_fork) {
    BLS_CUDA(cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming));
    for (int i = 0; i < 3; ++i) {
      BLS_CUDA(cudaStreamCreateWithFlags(&P->side[i], cudaStreamNonBlocking));
      BLS_CUDA(cudaEventCreateWithFlags(&P->ev_join[i], cudaEventDisableTiming));
    }
  }
  BLS_CUDA(cudaEventRecord(P->ev_fork, s));
  for (int i = 0; i < 3; ++i) BLS_CUDA(cudaStreamWaitEvent(P->side[i], P->ev_fork, 0));
}
static cudaStream_t class_stream(QRPlan* P, cudaStream_t s, int q) { return (q & 3) == 0 ? s : P->side[(q & 3) - 1]; }
static void join_sides(QRPlan* P, cudaStream_t s) {
  for (int i = 0; i < 3; ++i) {
    BLS_CUDA(cudaEventRecord(P->ev_join[i], P->side[i]));
    BLS_CUDA(cudaStreamWaitEvent(s, P->ev_join[i], 0));
  }
}

// Asynchronous global -> shared copies of one element (cp.async, completed by cp_async_wait_all): a lane issues all of
// its copies back to back, so a table's loads are in flight together instead of one DRAM latency per element.
template <class T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (sizeof(T) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// status: [0] lowest failing table, [1] lowest bad scaling_e entry
__global__ void k_qr_begin(long long* st) { st[0] = QNONE; st[1] = QNONE; st[2] = QNONE; }
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
// the sum over a group of G lanes (G a power of two up to 32, the group's lanes in gmask)
template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned gmask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o);
  return v;
}
// N independent sums over the group at once (each the same butterfly as group_sum; the N shuffles of a round overlap)
template <int G, int N>
__device__ __forceinline__ void group_sum_n(double (&v)[N], unsigned gmask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1)
#pragma unroll
    for (int n = 0; n < N; ++n) v[n] += __shfl_xor_sync(gmask, v[n], o);
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

// Eliminated blocks of up to QR_WY_MAX variables are factored in the compact form below; larger ones reflector by
// reflector.
constexpr int QR_WY_MAX = 4;

// Row i of the packed reflectors (QR_WY_MAX entries per row, those past the table's de zero): one 16-byte load in FP32,
// one or two in FP64.
template <class T, int ND>
__device__ __forceinline__ void load_vrow(const T* __restrict__ Vp, int i, T (&v)[QR_WY_MAX]) {
  if constexpr (sizeof(T) == 4) {
    const float4 x = reinterpret_cast<const float4*>(Vp)[i];
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    const double2* p = reinterpret_cast<const double2*>(Vp) + 2 * i;
    const double2 x = p[0];
    v[0] = x.x; v[1] = x.y;
    if constexpr (ND > 2) {
      const double2 y = p[1];
      v[2] = y.x; v[3] = y.y;
    } else {
      v[2] = T(0); v[3] = T(0);
    }
  }
}

// The ND reflectors H_k = I - tau_k v_k v_k' of a table applied to its retained columns in compact form: for a column y,
// H_{ND-1} ... H_0 y = y - V s with a = V' y and s_k = tau_k (a_k - sum_{l<k} s_l g_kl), g_kl = v_k' v_l, so each column
// is read twice (a, then the update) instead of twice per reflector. A lane per column; rows from me on are the
// damping rows, zero before the reflectors (read only for the non-finite test when `check`). V' y accumulates in the
// storage type, s in FP64. Returns whether a column held a non-finite entry (x * 0 is NaN exactly for Inf and NaN).
template <class T, int ND>
__device__ __forceinline__ bool wy_columns(T* A, const T* __restrict__ Vp, int ncols, int M, int me, const double* tau,
                                           const double* gkl, bool check, int lane, int G) {
  T chk = T(0);
  for (int j = lane; j < ncols; j += G) {
    T* y = A + (size_t)j * M;
    T a[ND];
#pragma unroll
    for (int k = 0; k < ND; ++k) a[k] = T(0);
    for (int i = 0; i < me; ++i) {
      const T x = y[i];
      T v[QR_WY_MAX];
      load_vrow<T, ND>(Vp, i, v);
      if (check) chk = fma(x, T(0), chk);
#pragma unroll
      for (int k = 0; k < ND; ++k) a[k] = fma(v[k], x, a[k]);
    }
    if (check)
      for (int i = me; i < M; ++i) chk = fma(y[i], T(0), chk);
    double sd[ND];
    T sv[ND];
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      double x = (double)a[k];
#pragma unroll
      for (int l = 0; l < k; ++l) x -= sd[l] * gkl[k * (k - 1) / 2 + l];
      sd[k] = tau[k] * x;
      sv[k] = T(-sd[k]);
    }
    for (int i = 0; i < me; ++i) {
      T v[QR_WY_MAX];
      load_vrow<T, ND>(Vp, i, v);
      T x = y[i];
#pragma unroll
      for (int k = 0; k < ND; ++k) x = fma(sv[k], v[k], x);
      y[i] = x;
    }
    for (int i = me; i < M; ++i) {
      T v[QR_WY_MAX];
      load_vrow<T, ND>(Vp, i, v);
      T x = sv[0] * v[0];
#pragma unroll
      for (int k = 1; k < ND; ++k) x = fma(sv[k], v[k], x);
      y[i] = x;
    }
  }
  return check && isnan((double)chk);
}

// The compact factorisation of a table whose eliminated block has ND <= QR_WY_MAX variables (its last ND columns, from
// ce): the eliminated columns' reflectors one after the other, each applied to the later eliminated columns (their dot
// products reduced together); then one pass over the rows packs V and forms the products g_kl = v_k'v_l and the
// residual's a = V'r (reduced together), a second updates the residual and clears the eliminated columns below their
// diagonal, and the retained columns take the compact update. Returns false when the table fails: a singular
// eliminated block, or a non-finite retained entry when `check`.
template <class T, int G, int ND>
__device__ __forceinline__ bool factor_wy(T* A, double* res, T* Vp, int M, int me, int ce, double tol, bool check, int lane,
                                          unsigned gmask) {
  double tau[ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    T* col = A + (ce + k) * M;
    // the column's norm above its diagonal (fewer than ND rows, read by every lane) and from its diagonal down
    double s_top = 0.0, s_sub = 0.0;
#pragma unroll
    for (int i = 0; i < k; ++i) {
      const double v = (double)col[i];
      s_top += v * v;
    }
    for (int i = k + lane; i < M; i += G) {
      const double v = (double)col[i];
      s_sub += v * v;
    }
    s_sub = group_sum<G>(s_sub, gmask);
    const double nrm = sqrt(s_sub), full = sqrt(s_top + s_sub);
    const double a = (double)col[k];
    const double beta = a >= 0.0 ? -nrm : nrm;
    if (!(isfinite(beta) && fabs(beta) > tol * full)) return false;
    const double scale = 1.0 / (a - beta);
    tau[k] = (beta - a) / beta;
    __syncwarp(gmask);   // every lane has read the column
    // the reflector's vector in place, and its products with the later eliminated columns
    double p[ND > 1 ? ND - 1 : 1];
#pragma unroll
    for (int n = 0; n < (ND > 1 ? ND - 1 : 1); ++n) p[n] = 0.0;
    for (int i = k + 1 + lane; i < M; i += G) {
      const T vt = T((double)col[i] * scale);
      col[i] = vt;
#pragma unroll
      for (int jj = k + 1; jj < ND; ++jj) p[jj - k - 1] += (double)vt * (double)A[(ce + jj) * M + i];
    }
    if (lane == 0) col[k] = T(beta);
    if (k + 1 < ND) {
      group_sum_n<G, (ND > 1 ? ND - 1 : 1)>(p, gmask);
      double q[ND > 1 ? ND - 1 : 1];
#pragma unroll
      for (int jj = k + 1; jj < ND; ++jj) q[jj - k - 1] = (p[jj - k - 1] + (double)A[(ce + jj) * M + k]) * tau[k];
      __syncwarp(gmask);   // every lane has read row k of the later columns
#pragma unroll
      for (int jj = k + 1; jj < ND; ++jj) {
        T* y = A + (ce + jj) * M;
        if (lane == 0) y[k] = T((double)y[k] - q[jj - k - 1]);
        for (int i = k + 1 + lane; i < M; i += G) y[i] = T((double)y[i] - q[jj - k - 1] * (double)col[i]);
      }
      __syncwarp(gmask);
    }
  }
  // V (v_k: zero above row k, one at row k, the stored vector below), g_kl and a = V'r
  constexpr int NG = ND * (ND - 1) / 2;
  double acc[NG + ND];
#pragma unroll
  for (int n = 0; n < NG + ND; ++n) acc[n] = 0.0;
  for (int i = lane; i < M; i += G) {
    T v[QR_WY_MAX];
#pragma unroll
    for (int k = 0; k < QR_WY_MAX; ++k) v[k] = k < ND ? (i < k ? T(0) : i == k ? T(1) : A[(ce + k) * M + i]) : T(0);
    if constexpr (sizeof(T) == 4) {
      reinterpret_cast<float4*>(Vp)[i] = make_float4(v[0], v[1], v[2], v[3]);
    } else {
      reinterpret_cast<double2*>(Vp)[2 * i] = make_double2(v[0], v[1]);
      reinterpret_cast<double2*>(Vp)[2 * i + 1] = make_double2(v[2], v[3]);
    }
    const double r = res[i];
#pragma unroll
    for (int k = 0; k < ND; ++k) {
#pragma unroll
      for (int l = 0; l < k; ++l) acc[k * (k - 1) / 2 + l] += (double)v[k] * (double)v[l];
      acc[NG + k] += (double)v[k] * r;
    }
  }
  group_sum_n<G, NG + ND>(acc, gmask);
  double sd[ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    double x = acc[NG + k];
#pragma unroll
    for (int l = 0; l < k; ++l) x -= sd[l] * acc[k * (k - 1) / 2 + l];
    sd[k] = tau[k] * x;
  }
  // the residual (rows over lanes, V from this lane's own rows) and the eliminated columns below their diagonal
  for (int i = lane; i < M; i += G) {
    double r = res[i];
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      r -= sd[k] * (double)Vp[QR_WY_MAX * i + k];
      if (i > k) A[(ce + k) * M + i] = T(0);
    }
    res[i] = r;
  }
  __syncwarp(gmask);   // V complete
  const bool bad = wy_columns<T, ND>(A, Vp, ce, M, me, tau, acc, check, lane, G);
  return !__any_sync(gmask, bad);
}

// qr_table! for the listed eliminated tables, a group of G lanes per table (G = 8 or 16 for narrow tables, so that a
// warp factors several tables at once and its lanes are not left idle over a few columns; 32 otherwise); the group's
// shared-memory region holds the table (M x C, column-major) and the FP64 residual (M). Tables are assigned by
// `tables[blockIdx.x * groups + group]`.
template <class T, int G>
__global__ void __launch_bounds__(32 * QR_MAX_WARPS, 8) k_qr_tables(int64_t ntab, int warp_bytes, const int32_t* __restrict__ tables,
                                                  const int32_t* __restrict__ t_rows,
                                                  const int32_t* __restrict__ t_cols, const int64_t* __restrict__ t_raw,
                                                  const int64_t* __restrict__ t_res, const int32_t* __restrict__ t_ptr,
                                                  const int32_t* __restrict__ u_col, const int32_t* __restrict__ u_ret,
                                                  const int32_t* __restrict__ boff_r, const int32_t* __restrict__ r_dims,
                                                  const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boff_e, int nr,
                                                  const T* __restrict__ Rw, const double* __restrict__ Rr, const double* __restrict__ sc_e,
                                                  double lambda, const double* __restrict__ s, T* __restrict__ F, double* __restrict__ Fr,
                                                  const T* __restrict__ Rw_end, const double* __restrict__ Rr_end, int bulk,
                                                  long long* st) {
  extern __shared__ __align__(16) unsigned char qsm_all[];
  // a group of G lanes per table (G = 8, 16 or 32, a warp holding 32 / G groups); gmask names the group's lanes
  const int grp = threadIdx.x / G;
  const int64_t wi = blockIdx.x * (int64_t)(blockDim.x / G) + grp;
  if (wi >= ntab) return;
  if (st[1] != QNONE) return;
  const int lane = threadIdx.x & (G - 1);
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (threadIdx.x & 31 & ~(G - 1)));
  unsigned char* qsm = qsm_all + (size_t)grp * warp_bytes;
  const int t = tables[wi];
  const int M = t_rows[t], C = t_cols[t] - 1, de = e_dims[t], me = M - de, ce = C - de;
  const int64_t off = t_raw[t], rq = t_res[t];
  // the group's region: its mbarrier, the packed reflectors of the compact form (M rows of QR_WY_MAX entries, when the
  // class left room for them), then the FP64 residual and the M x C table, each with 32 bytes of room for the 16-byte
  // alignment of a bulk copy
  uint64_t* bar = reinterpret_cast<uint64_t*>(qsm);
  const int rb = (8 * M + 32 + 15) & ~15, vb = QR_WY_MAX * (int)sizeof(T) * M;
  const bool wy = de <= QR_WY_MAX && 16 + vb + rb + (int64_t)sizeof(T) * M * C + 32 <= warp_bytes;
  T* Vp = reinterpret_cast<T*>(qsm + 16);
  unsigned char* rbase = qsm + 16 + (wy ? vb : 0);
  unsigned char* abase = rbase + rb;
  double* res;
  T* A;
  if (bulk & 1) {
    // the table and its residual are contiguous: one bulk copy each (TMA), completed on the group's mbarrier
    const Span sa = span_of(Rw + off, (int64_t)M * C, Rw_end), sr = span_of(Rr + rq, (int64_t)M, Rr_end);
    if (lane == 0) {
      mbar_init(bar, 1);
      mbar_fence_init();
      mbar_arrive_expect_tx(bar, span_bytes(sa) + span_bytes(sr));
      span_issue(reinterpret_cast<T*>(abase), sa, bar);
      span_issue(reinterpret_cast<double*>(rbase), sr, bar);
    }
    A = span_first(reinterpret_cast<T*>(abase), sa);
    res = span_first(reinterpret_cast<double*>(rbase), sr);
    __syncwarp(gmask);
    if (!mbar_wait(bar, 0)) {
      if (lane == 0) atomicExch(reinterpret_cast<unsigned long long*>(st + 2), 1ull);   // a copy that did not land: fault
      mbar_wait(bar, 0);                                                               // drain (bounded), then leave
      return;
    }
    __syncwarp(gmask);
  } else {
    res = reinterpret_cast<double*>(rbase);
    A = reinterpret_cast<T*>(abase);
    // element copies (coalesced: the table is contiguous; all of a lane's copies in flight at once)
    for (int i = lane; i < M * C; i += G) cp_async_elem(A + i, Rw + off + i);
    for (int i = lane; i < M; i += G) cp_async_elem(res + i, Rr + rq + i);
    cp_async_wait_all();
    __syncwarp(gmask);
  }
  // the reference's non-finite test (x - x is NaN for Inf / NaN) and the conditioning scales, in shared memory; in the
  // compact form without scales the retained columns are tested inside their update (before anything is written out)
  const bool fused = wy && !s;
  bool bad = false;
  for (int i = (fused ? ce * M : 0) + lane; i < M * C; i += G) {
    T x = A[i];
    bad |= isnan((double)(x - x));
    if (s) A[i] = T((double)x * col_scale(s, i / M, t, C, de, t_ptr, u_col, u_ret, boff_r, r_dims, boff_e, nr));
  }
  for (int i = lane; i < M; i += G) {
    const double x = res[i];
    bad |= isnan(x - x);
  }
  bad = __any_sync(gmask, bad);
  if (bad) {
    if (lane == 0) atomicMin(st, (long long)t);
    return;
  }
  __syncwarp(gmask);
  // damping rows: zero, with sqrt(lambda * scaling_e) * s_e (formed in FP64) on the eliminated columns' diagonal; the
  // compact form writes the retained columns' damping rows whole, so only the eliminated columns' are set for it
  const int z0 = wy ? ce : 0;
  for (int i = lane; i < de * (C - z0); i += G) {
    const int jj = i / de, r = i - jj * de, j = z0 + jj;
    T x = T(0);
    if (j - ce == r) {
      const int so = boff_e[t];
      x = T(sqrt(lambda * sc_e[so + r]) * (s ? s[nr + so + r] : 1.0));
    }
    A[j * M + me + r] = x;
  }
  for (int l = lane; l < de; l += G) res[me + l] = 0.0;
  __syncwarp(gmask);
  const double tol = (double)M * eps_of<T>();
  if (wy) {
    bool ok;
    if (de == 1) ok = factor_wy<T, G, 1>(A, res, Vp, M, me, ce, tol, fused, lane, gmask);
    else if (de == 2) ok = factor_wy<T, G, 2>(A, res, Vp, M, me, ce, tol, fused, lane, gmask);
    else if (de == 3) ok = factor_wy<T, G, 3>(A, res, Vp, M, me, ce, tol, fused, lane, gmask);
    else ok = factor_wy<T, G, 4>(A, res, Vp, M, me, ce, tol, fused, lane, gmask);
    if (!ok) {
      if (lane == 0) atomicMin(st, (long long)t);
      return;
    }
  } else {
    for (int k = 0; k < de; ++k) {
      T* col = A + (ce + k) * M;
      double s_top = 0.0, s_sub = 0.0;
      for (int i = lane; i < M; i += G) {
        const double v = (double)col[i];
        if (i < k) s_top += v * v;
        else s_sub += v * v;
      }
      s_top = group_sum<G>(s_top, gmask);
      s_sub = group_sum<G>(s_sub, gmask);
      const double nrm = sqrt(s_sub), full = sqrt(s_top + s_sub);
      const double a = (double)col[k];
      const double beta = a >= 0.0 ? -nrm : nrm;
      if (!(isfinite(beta) && fabs(beta) > tol * full)) {
        if (lane == 0) atomicMin(st, (long long)t);
        return;
      }
      const double scale = 1.0 / (a - beta);
      const double tau = (beta - a) / beta;
      __syncwarp(gmask);
      for (int i = k + 1 + lane; i < M; i += G) col[i] = T((double)col[i] * scale);
      __syncwarp(gmask);
      if (lane == 0) col[k] = T(beta);
      // apply I - tau v v' (v = [1; col[k+1:]]) to every column outside the eliminated columns ce..ce+k
      for (int j = lane; j < C; j += G) {
        if (j >= ce && j <= ce + k) continue;
        T* y = A + j * M;
        // v'y in four independent partial sums (the FMA chain is the latency of this loop), in the storage type: the
        // panel update is FP32 in the mixed form, the reflector's tau (its scaling) FP64
        T p0 = y[k], p1 = T(0), p2 = T(0), p3 = T(0);
        int i = k + 1;
        for (; i + 3 < M; i += 4) {
          p0 += col[i] * y[i];
          p1 += col[i + 1] * y[i + 1];
          p2 += col[i + 2] * y[i + 2];
          p3 += col[i + 3] * y[i + 3];
        }
        for (; i < M; ++i) p0 += col[i] * y[i];
        const T sj = T((double)((p0 + p1) + (p2 + p3)) * tau);
        y[k] = y[k] - sj;
        for (int i = k + 1; i < M; ++i) y[i] = y[i] - sj * col[i];
      }
      // and to the FP64 residual
      double sr = 0.0;
      for (int i = k + 1 + lane; i < M; i += G) sr += (double)col[i] * res[i];
      sr = group_sum<G>(sr, gmask) + res[k];
      sr *= tau;
      __syncwarp(gmask);
      if (lane == 0) res[k] -= sr;
      for (int i = k + 1 + lane; i < M; i += G) res[i] -= sr * (double)col[i];
      __syncwarp(gmask);
      for (int i = k + 1 + lane; i < M; i += G) col[i] = T(0);
      __syncwarp(gmask);
    }
  }
  __syncwarp(gmask);
  if (bulk & 2) {
    // the factored table out by one bulk copy of its aligned interior (F at the same 16-byte offset as the raw table)
    fence_proxy_async_shared();
    __syncwarp(gmask);
    if (lane == 0) span_store(F + off, A, (int64_t)M * C);
  } else {
    for (int i = lane; i < M * C; i += G) F[off + i] = A[i];
  }
  for (int i = lane; i < M; i += G) Fr[rq + i] = res[i];
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

// accumulate_qr_entry! (src/qr_reduced.jl:375-405) per table. MODE 0: S blocks (upper triangle of diagonal blocks) and
// J~'r~ into g; MODE 1: the full diagonal blocks D (reduced_diagonal_blocks!, :484-512). from_raw: the same products
// over the data rows of the raw tables, J'J of the retained columns and J'r (the retained part of the assembly).
template <class T, int MODE, bool ALL6>
__global__ void __launch_bounds__(32 * QR_MAX_WARPS) k_qr_gram(int64_t ntab, int warp_bytes, const int32_t* __restrict__ tables,
                                                              const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_cols,
                                                              const int32_t* __restrict__ t_top, const int64_t* __restrict__ t_raw,
                                                              const int64_t* __restrict__ t_res, const int32_t* __restrict__ t_ptr,
                                                              const int32_t* __restrict__ u_ret, const int32_t* __restrict__ u_col,
                                                              const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                                                              const int32_t* __restrict__ tp_ptr, const int32_t* __restrict__ tp_blk,
                                                              const int64_t* __restrict__ blk_base, const int32_t* __restrict__ blk_stride,
                                                              int64_t dense_nr, const int64_t* __restrict__ doff, int dmax, const T* __restrict__ F,
                                                              const double* __restrict__ Fr, T* __restrict__ S, double* __restrict__ g, int from_raw,
                                                              const T* __restrict__ F_end, const double* __restrict__ Fr_end, int bulk,
                                                              long long* st) {
  extern __shared__ __align__(16) unsigned char gsm_all[];
  const int64_t wi = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (wi >= ntab) return;
  const int lane = threadIdx.x & 31;
  unsigned char* gsm = gsm_all + (size_t)(threadIdx.x >> 5) * warp_bytes;
  const int t = tables[wi];
  const int M = t_rows[t], top = t_top[t], n = M - top, ce = t_cols[t] - 1 - top;
  const int u0 = t_ptr[t], kt = t_ptr[t + 1] - u0;
  // the warp's region: its mbarrier, the residual rows (FP64), then the retained columns
  uint64_t* bar = reinterpret_cast<uint64_t*>(gsm);
  unsigned char* rbase = gsm + 16;
  unsigned char* bbase = rbase + ((8 * n + 32 + 15) & ~15);
  double* rr;
  T* B;
  int ns;   // column stride of B in shared memory
  // rows [row0, row0 + n): the bottom rows J~ of a factored table, or the data rows of a raw one (its damping rows last)
  const int row0 = from_raw ? 0 : top;
  const T* src = F + t_raw[t] + row0;
  if (bulk && ce > 0) {
    // rows row0.. of columns 0..ce-1 lie in one contiguous span of (ce - 1) M + n entries: one bulk copy (TMA), the
    // columns then at stride M (the rows above row0 of columns 1.. come along and are not read)
    ns = M;
    const Span sb = span_of(src, (int64_t)(ce - 1) * M + n, F_end);
    const Span sr = span_of(Fr + t_res[t] + row0, (int64_t)n, Fr_end);
    if (lane == 0) {
      mbar_init(bar, 1);
      mbar_fence_init();
      mbar_arrive_expect_tx(bar, span_bytes(sb) + (MODE == 0 ? span_bytes(sr) : 0u));
      span_issue(reinterpret_cast<T*>(bbase), sb, bar);
      if (MODE == 0) span_issue(reinterpret_cast<double*>(rbase), sr, bar);
    }
    B = span_first(reinterpret_cast<T*>(bbase), sb);
    rr = span_first(reinterpret_cast<double*>(rbase), sr);
    __syncwarp();
    if (!mbar_wait(bar, 0)) {
      if (lane == 0) atomicExch(reinterpret_cast<unsigned long long*>(st + 2), 1ull);   // a copy that did not land: fault
      mbar_wait(bar, 0);
      return;
    }
    __syncwarp();
  } else {
    ns = n | 1;
    rr = reinterpret_cast<double*>(rbase);
    B = reinterpret_cast<T*>(bbase);
    for (int q = lane; q < ce * n; q += 32) {
      const int j = q / n, i = q - j * n;
      cp_async_elem(B + j * ns + i, src + (int64_t)j * M + i);
    }
    if (MODE == 0)
      for (int i = lane; i < n; i += 32) cp_async_elem(rr + i, Fr + t_res[t] + row0 + i);
    cp_async_wait_all();
    __syncwarp();
  }
  if (MODE == 0) {
    // J~'r~: lane per column, entry found by scanning the table's entries
    for (int j = lane; j < ce; j += 32) {
      int gi = 0;
      for (int u = u0; u < u0 + kt; ++u) {
        const int c0 = u_col[u], r = u_ret[u];
        if (j >= c0 && j < c0 + r_dims[r]) gi = boff_r[r] + (j - c0);
      }
      double acc = 0.0;
      for (int i = 0; i < n; ++i) acc += (double)B[j * ns + i] * rr[i];
      atomicAdd(g + gi, acc);
    }
  }
  // From the raw tables (the assembly), an entry's columns are zero outside its own observations' rows in a
  // bundle-adjustment table: each entry's nonzero row span [lo, hi) bounds its products, and a pair whose spans do not
  // meet adds nothing (the output was zeroed). The spans go to rr once J'r is done; a table with more entries than rr
  // has slots keeps the full range.
  const int2* span = nullptr;
  if (from_raw && kt <= ((n + 1) & ~1)) {
    __syncwarp();
    int2* sp = reinterpret_cast<int2*>(rr);
    for (int ul = lane; ul < kt; ul += 32) {
      const int c0 = u_col[u0 + ul], d = r_dims[u_ret[u0 + ul]];
      int lo = n, hi = 0;
      for (int i = 0; i < n; ++i) {
        bool nz = false;
        for (int a = 0; a < d; ++a) nz |= B[(c0 + a) * ns + i] != T(0);
        if (nz) {
          lo = min(lo, i);
          hi = i + 1;
        }
      }
      sp[ul] = make_int2(lo, hi);
    }
    __syncwarp();
    span = sp;
  }
  // work units: (pair, a group of three columns of the pair's block); lanes take units in order, so the lanes of one
  // pair read the same X rows (shared-memory broadcast)
  const int npairs = kt * (kt + 1) / 2;
  constexpr int G = 3;   // columns of the pair's block per work unit
  const int upp = (dmax + G - 1) / G;
  for (int q = lane; q < npairs * upp; q += 32) {
    const int p = q / upp, w0 = G * (q - p * upp);
    int u2l = (int)((sqrtf(8.0f * p + 1.0f) - 1.0f) * 0.5f);
    while ((u2l + 1) * (u2l + 2) / 2 <= p) ++u2l;
    while (u2l * (u2l + 1) / 2 > p) --u2l;
    const int u1l = p - u2l * (u2l + 1) / 2;
    const bool diag = u1l == u2l;
    if (MODE == 1 && !diag) continue;
    const int r1 = u_ret[u0 + u1l], r2 = u_ret[u0 + u2l];
    const int d1 = r_dims[r1], d2 = r_dims[r2];
    if (w0 >= d2) continue;
    const int ilo = span ? max(span[u1l].x, span[u2l].x) : 0, ihi = span ? min(span[u1l].y, span[u2l].y) : n;
    if (ilo >= ihi) continue;
    const T* X = B + u_col[u0 + u1l] * ns;
    const T* Y = B + (u_col[u0 + u2l] + w0) * ns;
    T* out;
    int64_t stride;
    if (MODE == 0) {
      const int k = tp_blk[tp_ptr[t] + p];
      stride = blk_stride ? (int64_t)blk_stride[k] : dense_nr;
      out = S + blk_base[k] + w0 * stride;
    } else {
      stride = d2;
      out = S + doff[r2] + w0 * d2;
    }
    if (ALL6 || (d1 == 6 && d2 == 6)) {
      // products accumulated in the storage type: FP32 in the mixed form (the bulk of the arithmetic), FP64 otherwise
      T acc[G][6];
#pragma unroll
      for (int w = 0; w < G; ++w)
#pragma unroll
        for (int a = 0; a < 6; ++a) acc[w][a] = T(0);
      for (int i = ilo; i < ihi; ++i) {
        T x[6], y[G];
#pragma unroll
        for (int a = 0; a < 6; ++a) x[a] = X[a * ns + i];
#pragma unroll
        for (int w = 0; w < G; ++w) y[w] = Y[w * ns + i];
#pragma unroll
        for (int w = 0; w < G; ++w)
#pragma unroll
          for (int a = 0; a < 6; ++a) acc[w][a] += x[a] * y[w];
      }
#pragma unroll
      for (int w = 0; w < G; ++w)
#pragma unroll
        for (int a = 0; a < 6; ++a)
          if (MODE == 1 || !diag || a <= w0 + w) atomicAdd(out + w * stride + a, acc[w][a]);
    } else if (!ALL6) {
      for (int w = w0; w < d2 && w < w0 + G; ++w) {
        double acc[16];
#pragma unroll
        for (int a = 0; a < 16; ++a) acc[a] = 0.0;
        for (int i = ilo; i < ihi; ++i) {
          const double y = (double)Y[(w - w0) * ns + i];
#pragma unroll
          for (int a = 0; a < 16; ++a)
            if (a < d1) acc[a] += (double)X[a * ns + i] * y;
        }
#pragma unroll
        for (int a = 0; a < 16; ++a)
          if (a < d1 && (MODE == 1 || !diag || a <= w)) atomicAdd(out + (w - w0) * stride + a, T(acc[a]));
      }
    }
  }
}

// The eliminated part of H = J'J, b = J'r from the raw tables (no device counterpart in the reference, whose callers
// fill a SchurBlockHessian block by block with addblock!, src/schur_assembly.jl:140-246; the reference's own fixtures
// form J'J in FP64 and round it once, test/fixtures/QRFixtures.jl:109-120): one warp per eliminated table, sums over
// its data rows (the first M - d_e; the damping rows are last) accumulated in FP64 and rounded once. E_e (d_e x d_e,
// column-major at the point's E offset), b_e, and per entry the coupling block, d_e x d_r column-major at its C offset
// (entry (a, w) = sum_i J[i, point col a] J[i, entry col w], add_coupling!'s transposed storage). Each table owns its
// outputs, so every entry is written once.
template <class T>
__global__ void __launch_bounds__(128) k_qr_point_gram(int64_t neb, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_cols,
                                                       const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_res,
                                                       const int32_t* __restrict__ t_ptr, const int32_t* __restrict__ u_ret,
                                                       const int32_t* __restrict__ u_col, const int32_t* __restrict__ r_dims,
                                                       const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boff_e,
                                                       const int64_t* __restrict__ t_eoff, const int64_t* __restrict__ u_coff,
                                                       const T* __restrict__ J, const double* __restrict__ res, T* __restrict__ E,
                                                       T* __restrict__ Cd, double* __restrict__ b_e) {
  const int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= neb) return;
  const int M = t_rows[e], de = e_dims[e], n = M - de, ce = t_cols[e] - 1 - de;
  const T* tab = J + t_raw[e];
  const T* P = tab + (int64_t)ce * M;   // the point's columns
  const double* rr = res + t_res[e];
  for (int q = lane; q < de * de + de; q += 32) {
    double acc = 0.0;
    if (q < de * de) {
      const T* x = P + (int64_t)(q % de) * M;
      const T* y = P + (int64_t)(q / de) * M;
      for (int i = 0; i < n; ++i) acc += (double)x[i] * (double)y[i];
      E[t_eoff[e] + q] = T(acc);
    } else {
      const T* x = P + (int64_t)(q - de * de) * M;
      for (int i = 0; i < n; ++i) acc += (double)x[i] * rr[i];
      b_e[boff_e[e] + (q - de * de)] = acc;
    }
  }
  for (int u = t_ptr[e]; u < t_ptr[e + 1]; ++u) {
    const int dr = r_dims[u_ret[u]];
    const T* Y = tab + (int64_t)u_col[u] * M;
    for (int q = lane; q < de * dr; q += 32) {
      const int a = q % de, w = q / de;
      const T* x = P + (int64_t)a * M;
      const T* y = Y + (int64_t)w * M;
      double acc = 0.0;
      for (int i = 0; i < n; ++i) acc += (double)x[i] * (double)y[i];
      Cd[u_coff[u] + q] = T(acc);
    }
  }
}

// Quantities of the full problem from the raw or the factored tables (src/qr_reduced.jl:515-640), every row of each
// table, FP64 accumulation. MODE 0, jtr! (:575-584): g = [J'r over the retained columns, summed per block; J'r over each
// point's columns]. MODE 1, jtj_diag! (:586-595): the squared column norms. Retained part: one warp per retained
// block, lanes over its entries (sum_retained_columns!, :536-560), then a butterfly sum.
__device__ __forceinline__ double warp_sum_q(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <class T, int MODE>
__global__ void __launch_bounds__(256) k_jt_retained(int64_t nrb, const int32_t* __restrict__ rptr, const int32_t* __restrict__ rent,
                                                     const int32_t* __restrict__ u_tab, const int32_t* __restrict__ u_col,
                                                     const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                                                     const int32_t* __restrict__ t_rows, const int64_t* __restrict__ t_raw,
                                                     const int64_t* __restrict__ t_res, const T* __restrict__ D,
                                                     const double* __restrict__ Rv, double* __restrict__ out) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= nrb) return;
  const int dr = r_dims[r];
  double acc[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) acc[j] = 0.0;
  for (int k = rptr[r] + lane; k < rptr[r + 1]; k += 32) {
    const int u = rent[k], t = u_tab[u], M = t_rows[t];
    const T* cb = D + t_raw[t] + (int64_t)u_col[u] * M;
    const double* rb = Rv + t_res[t];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      if (j >= dr) break;
      const T* c = cb + (int64_t)j * M;
      double a = 0.0;
      for (int i = 0; i < M; ++i) a += MODE == 0 ? (double)c[i] * rb[i] : (double)c[i] * (double)c[i];
      acc[j] += a;
    }
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) acc[j] = warp_sum_q(acc[j]);
  if (lane < dr) {
    double v = 0.0;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (j == lane) v = acc[j];
    out[boff_r[r] + lane] = v;
  }
}
// The eliminated part: thread per eliminated table, its d_e point columns (foreach_eliminated_column, :562-573)
template <class T, int MODE>
__global__ void k_jt_eliminated(int64_t neb, int64_t nr, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_cols,
                                const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_res, const int32_t* __restrict__ e_dims,
                                const int32_t* __restrict__ boff_e, const T* __restrict__ D, const double* __restrict__ Rv,
                                double* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb) return;
  const int M = t_rows[e], C = t_cols[e], de = e_dims[e];
  for (int k = 0; k < de; ++k) {
    const T* c = D + t_raw[e] + (int64_t)(C - de - 1 + k) * M;
    const double* rb = Rv + t_res[e];
    double a = 0.0;
    for (int i = 0; i < M; ++i) a += MODE == 0 ? (double)c[i] * rb[i] : (double)c[i] * (double)c[i];
    out[nr + boff_e[e] + k] = a;
  }
}
// jtj_quadform (:597-640): ||J v||^2 = sum over tables and rows of (row . v)^2, FP64. One warp per table, lanes over
// rows; each table's part is added to one FP64 accumulator.
template <class T>
__global__ void __launch_bounds__(256) k_jtj_quadform(int64_t nt, int64_t neb, int64_t nr, const int32_t* __restrict__ t_rows,
                                                      const int32_t* __restrict__ t_cols, const int64_t* __restrict__ t_raw,
                                                      const int32_t* __restrict__ t_ptr, const int32_t* __restrict__ u_ret,
                                                      const int32_t* __restrict__ u_col, const int32_t* __restrict__ r_dims,
                                                      const int32_t* __restrict__ boff_r, const int32_t* __restrict__ e_dims,
                                                      const int32_t* __restrict__ boff_e, const T* __restrict__ D,
                                                      const double* __restrict__ v, double* __restrict__ total) {
  const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= nt) return;
  const int M = t_rows[t], C = t_cols[t];
  const int de = t < neb ? e_dims[t] : 0;
  const T* tab = D + t_raw[t];
  double part = 0.0;
  for (int i = lane; i < M; i += 32) {
    double y = 0.0;
    for (int u = t_ptr[t]; u < t_ptr[t + 1]; ++u) {
      const int r = u_ret[u], ro = boff_r[r];
      const T* cb = tab + (int64_t)u_col[u] * M + i;
      for (int j = 0; j < r_dims[r]; ++j) y += (double)cb[(int64_t)j * M] * v[ro + j];
    }
    if (de) {
      const T* cb = tab + (int64_t)(C - de - 1) * M + i;
      const int64_t eo = nr + boff_e[t];
      for (int k = 0; k < de; ++k) y += (double)cb[(int64_t)k * M] * v[eo + k];
    }
    part += y * y;
  }
  part = warp_sum_q(part);
  if (lane == 0 && part != 0.0) atomicAdd(total, part);
}

// qr_backsubstitute_group! (src/qr_reduced.jl:24-93): thread per eliminated table, FP64
template <class T>
__global__ void k_qr_backsub(int64_t ne_tab, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_cols,
                             const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_res, const int32_t* __restrict__ t_ptr,
                             const int32_t* __restrict__ u_col, const int32_t* __restrict__ u_ret, const int32_t* __restrict__ r_dims,
                             const int32_t* __restrict__ boff_r, const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boff_e,
                             const T* __restrict__ F, const double* __restrict__ Fr, const double* __restrict__ x_r, double* __restrict__ x_e,
                             const double* __restrict__ w = nullptr) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne_tab) return;
  const int M = t_rows[e], C = t_cols[e], de = e_dims[e], ce = C - de - 1;
  const int64_t off = t_raw[e];
  // t = q - B x_r accumulated in x_e's own entries, then U x_e = t solved in place (the same operations in the same order);
  // q is the factored residual's top rows, or the given w (a refinement step's U^-T d_e)
  double* xe = x_e + boff_e[e];
  for (int i = 0; i < de; ++i) xe[i] = w ? w[boff_e[e] + i] : Fr[t_res[e] + i];
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

// Iterative refinement of the QR route (no reference counterpart; the reference solves the reduced system once,
// src/qr_linear_systems.jl:250-300). A step needs the normal-equation residual of the whole damped problem in FP64 and
// the reduction of that residual through the factored tables:
//   y = r - J x on every row of the raw tables (the damping rows of an eliminated table are zero: its damping is
//       lambda * scaling, added below), then d = J' y - lambda * scaling .* x (d through jtr!'s kernels);
//   per eliminated table, with its factored top rows [U B]: w = U^-T d_e and d_r -= B' w, so that the correction of x_r
//       solves (J~'J~ + lambda diag(scaling_r)) dx_r = d_r, and dx_e = U^-1 (w - B dx_r) (the back-substitution with w).
// U' U and U' B are the eliminated and coupling blocks of J'J + lambda diag(scaling) (the table's QR), so the three
// steps are the block elimination of the normal equations with the factored tables; everything is FP64 arithmetic on
// the tables' storage type.
template <class T>
__global__ void __launch_bounds__(256) k_qr_rows_residual(int64_t ntab, int64_t neb, const int32_t* __restrict__ t_rows,
                                                          const int32_t* __restrict__ t_cols, const int64_t* __restrict__ t_raw,
                                                          const int64_t* __restrict__ t_res, const int32_t* __restrict__ t_ptr,
                                                          const int32_t* __restrict__ u_col, const int32_t* __restrict__ u_ret,
                                                          const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                                                          const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boff_e, int64_t nr,
                                                          const T* __restrict__ J, const double* __restrict__ r, const double* __restrict__ x,
                                                          double* __restrict__ y) {
  const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= ntab) return;
  const int M = t_rows[t], C = t_cols[t] - 1;
  const bool elim = t < neb;
  const int de = elim ? e_dims[t] : 0, me = M - de, ce = C - de;
  const int64_t off = t_raw[t], rq = t_res[t];
  for (int i = lane; i < M; i += 32) {
    if (i >= me) {   // an eliminated table's damping rows
      y[rq + i] = 0.0;
      continue;
    }
    double acc = r[rq + i];
    for (int u = t_ptr[t]; u < t_ptr[t + 1]; ++u) {
      const int c0 = u_col[u], ro = boff_r[u_ret[u]], d = r_dims[u_ret[u]];
      for (int j = 0; j < d; ++j) acc -= (double)J[off + (int64_t)(c0 + j) * M + i] * x[ro + j];
    }
    for (int j = 0; j < de; ++j) acc -= (double)J[off + (int64_t)(ce + j) * M + i] * x[nr + boff_e[t] + j];
    y[rq + i] = acc;
  }
}

__global__ void k_sub_damping(int64_t n, double lambda, const double* __restrict__ sc, const double* __restrict__ x, double* __restrict__ d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) d[i] -= lambda * sc[i] * x[i];
}

template <class T>
__global__ void __launch_bounds__(128) k_qr_reduce_rhs(int64_t neb, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_cols,
                                                       const int64_t* __restrict__ t_raw, const int32_t* __restrict__ t_ptr,
                                                       const int32_t* __restrict__ u_col, const int32_t* __restrict__ u_ret,
                                                       const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                                                       const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boff_e, int64_t nr,
                                                       const T* __restrict__ F, const double* __restrict__ d, double* __restrict__ w,
                                                       double* __restrict__ d_r) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb) return;
  const int M = t_rows[e], C = t_cols[e] - 1, de = e_dims[e], ce = C - de;
  const int64_t off = t_raw[e];
  double we[16];
  for (int i = 0; i < de; ++i) {   // U' w = d_e, forward substitution (U upper triangular in the top rows)
    double acc = d[nr + boff_e[e] + i];
    for (int k = 0; k < i; ++k) acc -= (double)F[off + (int64_t)(ce + i) * M + k] * we[k];
    we[i] = acc / (double)F[off + (int64_t)(ce + i) * M + i];
    w[boff_e[e] + i] = we[i];
  }
  for (int u = t_ptr[e]; u < t_ptr[e + 1]; ++u) {   // d_r -= B' w
    const int c0 = u_col[u], ro = boff_r[u_ret[u]], dr = r_dims[u_ret[u]];
    for (int j = 0; j < dr; ++j) {
      double acc = 0.0;
      for (int i = 0; i < de; ++i) acc += (double)F[off + (int64_t)(c0 + j) * M + i] * we[i];
      atomicAdd(d_r + ro + j, -acc);
    }
  }
}

template <class T>
__global__ void k_fill_t(T* __restrict__ p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = T(0);
}

// ------------------------------------------------------------------------------------------------------------------
// Plan
// ------------------------------------------------------------------------------------------------------------------
// reduced_residual! (src/qr_reduced.jl:227-243): r~, a warp per table copying its bottom residual rows
__global__ void __launch_bounds__(256) k_reduced_residual(int64_t nt, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_top,
                                                          const int64_t* __restrict__ t_res, const int64_t* __restrict__ t_red,
                                                          const double* __restrict__ Fr, double* __restrict__ rt) {
  const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= nt) return;
  const int n = t_rows[t] - t_top[t];
  const double* src = Fr + t_res[t] + t_top[t];
  double* dst = rt + t_red[t];
  for (int i = lane; i < n; i += 32) dst[i] = src[i];
}

// reduced_jacobian!(Jt::Matrix, ...) (src/qr_reduced.jl:245-272): a warp per table writes the bottom rows of each
// entry's columns of the factored table into J~ (column-major, leading dimension ld = reduced_nrows; zeroed before)
template <class T>
__global__ void __launch_bounds__(256) k_reduced_jacobian_dense(int64_t nt, const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_top,
                                                                const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_red,
                                                                const int32_t* __restrict__ t_ptr, const int32_t* __restrict__ u_ret,
                                                                const int32_t* __restrict__ u_col, const int32_t* __restrict__ r_dims,
                                                                const int32_t* __restrict__ boff_r, const T* __restrict__ F, T* __restrict__ Jt,
                                                                int64_t ld) {
  const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= nt) return;
  const int M = t_rows[t], top = t_top[t], n = M - top;
  const int64_t raw = t_raw[t], red = t_red[t];
  for (int u = t_ptr[t]; u < t_ptr[t + 1]; ++u) {
    const int r = u_ret[u], dr = r_dims[r], c0 = u_col[u];
    const int64_t ro = boff_r[r];
    for (int q = lane; q < dr * n; q += 32) {
      const int j = q / n, i = q - j * n;
      Jt[(red + i) + ld * (ro + j)] = F[raw + (int64_t)(c0 + j) * M + top + i];
    }
  }
}

// reduced_jacobian!(Jt::SparseMatrixCSC, ...) (src/qr_reduced.jl:336-370): a warp per entry writes its run of
// bottom rows into every column of its retained block, at the run's position in the column
template <class T>
__global__ void __launch_bounds__(256) k_reduced_jacobian_sparse(int64_t nent, const int32_t* __restrict__ u_tab, const int32_t* __restrict__ t_rows,
                                                                 const int32_t* __restrict__ t_top, const int64_t* __restrict__ t_raw,
                                                                 const int32_t* __restrict__ u_ret, const int32_t* __restrict__ u_col,
                                                                 const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                                                                 const int64_t* __restrict__ jt_colptr, const int64_t* __restrict__ u_runpos,
                                                                 const T* __restrict__ F, T* __restrict__ nzval) {
  const int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (u >= nent) return;
  const int t = u_tab[u], M = t_rows[t], top = t_top[t], n = M - top, r = u_ret[u], dr = r_dims[r];
  const int64_t ro = boff_r[r], cb = t_raw[t] + (int64_t)u_col[u] * M + top, p = u_runpos[u];
  for (int q = lane; q < dr * n; q += 32) {
    const int j = q / n, i = q - j * n;
    nzval[jt_colptr[ro + j] + p + i] = F[cb + (int64_t)j * M + i];
  }
}

template <class T>
static void reduced_jacobian_dense(QRPlan* P, T* Jt, const T* F, const double* Fr, double* rt) {
  cudaStream_t s = P->ctx->stream;
  const int64_t m = P->red_nrows;
  if (m > 0) BLS_CUDA(cudaMemsetAsync(Jt, 0, sizeof(T) * (size_t)m * (size_t)P->nr, s));
  const unsigned g = (unsigned)std::max(1, grid_for(P->ntables * 32, 256));
  k_reduced_residual<<<g, 256, 0, s>>>(P->ntables, P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_res.as<int64_t>(), P->t_red.as<int64_t>(), Fr, rt);
  k_reduced_jacobian_dense<T><<<g, 256, 0, s>>>(P->ntables, P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(),
                                                P->t_red.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_ret.as<int32_t>(), P->u_col.as<int32_t>(),
                                                P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), F, Jt, m);
  P->launches += 2;
  BLS_CUDA(cudaGetLastError());
}

template <class T>
static void reduced_jacobian_sparse(QRPlan* P, T* nzval, const T* F, const double* Fr, double* rt) {
  cudaStream_t s = P->ctx->stream;
  k_reduced_residual<<<(unsigned)std::max(1, grid_for(P->ntables * 32, 256)), 256, 0, s>>>(
      P->ntables, P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_res.as<int64_t>(), P->t_red.as<int64_t>(), Fr, rt);
  if (P->nentries > 0)
    k_reduced_jacobian_sparse<T><<<(unsigned)grid_for(P->nentries * 32, 256), 256, 0, s>>>(
        P->nentries, P->u_tab.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(), P->u_ret.as<int32_t>(),
        P->u_col.as<int32_t>(), P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), P->jt_colptr.as<int64_t>(), P->u_runpos.as<int64_t>(), F, nzval);
  P->launches += 2;
  BLS_CUDA(cudaGetLastError());
}

// reduced_mul! (src/qr_reduced.jl:159-192): y = J~ v, a thread per reduced row (its table from red_tab, so that warps
// run across table boundaries rather than idling lanes past a table's few rows), accumulating over the table's entries
// and their columns in order (FP64)
template <class T>
__global__ void __launch_bounds__(256) k_reduced_mul(int64_t nrows, const int32_t* __restrict__ red_tab, const int32_t* __restrict__ t_rows,
                                                     const int32_t* __restrict__ t_top, const int64_t* __restrict__ t_raw,
                                                     const int64_t* __restrict__ t_red, const int32_t* __restrict__ t_ptr,
                                                     const int32_t* __restrict__ u_ret, const int32_t* __restrict__ u_col,
                                                     const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                                                     const T* __restrict__ F, const double* __restrict__ v, double* __restrict__ y) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  const int t = red_tab[row];
  const int M = t_rows[t], top = t_top[t];
  const int64_t raw = t_raw[t] + top + (row - t_red[t]);
  const int u0 = t_ptr[t], u1 = t_ptr[t + 1];
  double acc = 0.0;
  for (int u = u0; u < u1; ++u) {
    const int r = u_ret[u], dr = r_dims[r], c0 = u_col[u], ro = boff_r[r];
    const T* col = F + raw + (int64_t)c0 * M;
    if (dr == 6) {   // the common camera block: six independent loads in flight
      T f[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) f[j] = col[(int64_t)j * M];
#pragma unroll
      for (int j = 0; j < 6; ++j) acc += (double)f[j] * v[ro + j];
    } else {
      for (int j = 0; j < dr; ++j) acc += (double)col[(int64_t)j * M] * v[ro + j];
    }
  }
  y[row] = acc;
}

// reduced_tmul! (src/qr_reduced.jl:194-223): g = J~' w in two passes, so that the work spreads over every entry rather
// than one warp per retained block (a few hundred warps on a bundle-adjustment scene, each walking thousands of runs
// in sequence). Pass 1, a thread per (entry, column): the dot product of the entry's run in that column with w, FP64,
// into part[u * dmax + j]. Pass 2, a warp per (retained block, column): the sum over the block's entries in their order
// (lanes strided, then a butterfly), written to g. Deterministic: no atomics.
template <class T>
__global__ void __launch_bounds__(256) k_tmul_entries(int64_t nent, int dmax, const int4* __restrict__ meta,
                                                      const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_top,
                                                      const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_red,
                                                      const T* __restrict__ F, const double* __restrict__ w,
                                                      double* __restrict__ part) {
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= nent * dmax) return;
  const int64_t u = gid / dmax;
  const int j = (int)(gid - u * dmax);
  const int4 q = meta[u];   // column, retained offset, retained size, table
  if (j >= q.z) return;
  const int t = q.w, M = t_rows[t], top = t_top[t], n = M - top;
  const T* col = F + t_raw[t] + (int64_t)(q.x + j) * M + top;
  const double* wr = w + t_red[t];
  double acc = 0.0;
#pragma unroll 4
  for (int i = 0; i < n; ++i) acc += (double)col[i] * wr[i];
  part[gid] = acc;
}

__global__ void __launch_bounds__(256) k_tmul_reduce(int64_t nrb, int dmax, const int32_t* __restrict__ rptr,
                                                     const int32_t* __restrict__ rent, const int32_t* __restrict__ r_dims,
                                                     const int32_t* __restrict__ boff_r, const double* __restrict__ part,
                                                     double* __restrict__ g) {
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t r = gw / dmax;
  const int j = (int)(gw - r * dmax);
  if (r >= nrb || j >= r_dims[r]) return;   // uniform across the warp
  double acc = 0.0;
  for (int k = rptr[r] + lane; k < rptr[r + 1]; k += 32) acc += part[(int64_t)rent[k] * dmax + j];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) g[boff_r[r] + j] = acc;
}

template <class T>
static void launch_reduced_mul(QRPlan* P, const T* F, const double* v, double* y) {
  if (P->red_nrows == 0) return;
  k_reduced_mul<T><<<(unsigned)grid_for(P->red_nrows, 256), 256, 0, P->ctx->stream>>>(
      P->red_nrows, P->red_tab.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(), P->t_red.as<int64_t>(),
      P->t_ptr.as<int32_t>(), P->u_ret.as<int32_t>(), P->u_col.as<int32_t>(), P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), F, v, y);
  P->launches += 1;
  BLS_CUDA(cudaGetLastError());
}

template <class T>
static void launch_reduced_tmul(QRPlan* P, const T* F, const double* w, double* g) {
  cudaStream_t s = P->ctx->stream;
  if (P->rdmax == 0)
    for (int64_t d : P->h_rdims) P->rdmax = std::max<int>(P->rdmax, (int)d);
  const int dm = std::max(P->rdmax, 1);
  const size_t need = sizeof(double) * (size_t)std::max<int64_t>(P->nentries * dm, 1);
  if (P->tm_part.bytes < need) P->tm_part.alloc(need);
  double* part = P->tm_part.as<double>();
  if (P->nentries > 0)
    k_tmul_entries<T><<<(unsigned)grid_for(P->nentries * dm, 256), 256, 0, s>>>(
        P->nentries, dm, P->u_meta.as<int4>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(),
        P->t_red.as<int64_t>(), F, w, part);
  k_tmul_reduce<<<(unsigned)std::max(1, grid_for(P->nrblocks * dm * 32, 256)), 256, 0, s>>>(
      P->nrblocks, dm, P->q_rptr.as<int32_t>(), P->q_rent.as<int32_t>(), P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), part, g);
  P->launches += 1 + (P->nentries > 0);
  BLS_CUDA(cudaGetLastError());
}

// check_reduced_jacobian_pattern (src/qr_reduced.jl:312-334) of a caller's 0-based CSC, before any work: its size,
// then per column of each retained block its height and the first row of every run; messages 1-based, as the
// reference's
static void check_jt_pattern(const QRPlan* P, int64_t nrows, int64_t ncols, const int64_t* colptr, const int64_t* rowval) {
  if (nrows != P->red_nrows || ncols != P->nr)
    throw Error(BLS_EDIM, "Jt has size (" + std::to_string(nrows) + ", " + std::to_string(ncols) + "), expected (" + std::to_string(P->red_nrows) +
                              ", " + std::to_string(P->nr) + ")");
  if (!colptr) throw Error(BLS_EINVAL, "the pattern of Jt is NULL");
  for (int64_t r = 0; r < P->nrblocks; ++r)
    for (int64_t c = P->h_boff_r[r]; c < P->h_boff_r[r] + P->h_rdims[r]; ++c) {
      const int64_t h = P->h_jt_colptr[c + 1] - P->h_jt_colptr[c];
      if (colptr[c + 1] - colptr[c] != h)
        throw Error(BLS_EINVAL, "Jt does not have the pattern of build_reduced_jacobian_pattern: column " + std::to_string(c + 1) + " stores " +
                                    std::to_string(colptr[c + 1] - colptr[c]) + " entries, expected " + std::to_string(h));
      int64_t p = colptr[c];
      for (int32_t k = P->h_rptr[r]; k < P->h_rptr[r + 1]; ++k) {
        const int32_t t = P->h_rent_tab[k];
        const int64_t n = P->h_red[t + 1] - P->h_red[t];
        if (n != 0 && (!rowval || rowval[p] != P->h_red[t]))
          throw Error(BLS_EINVAL, "Jt does not have the pattern of build_reduced_jacobian_pattern: column " + std::to_string(c + 1) +
                                      " stores row " + (rowval ? std::to_string(rowval[p] + 1) : std::string("?")) + ", expected " +
                                      std::to_string(P->h_red[t] + 1));
        p += n;
      }
    }
}

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
    if (d->r_dims[r] != 6) P->all6 = false;
  }
  for (int64_t e = 0; e < neb; ++e) {
    if (d->e_dims[e] < 1) throw Error(BLS_EINVAL, "eliminated block sizes must be positive");
    P->max_de = std::max<int>(P->max_de, (int)std::min<int64_t>(d->e_dims[e], 1 << 20));
    boff_e[e] = ne; ne += d->e_dims[e];
  }
  P->nr = nr; P->ne = ne;
  P->ndiag = doff[nrb];
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
  // shared-memory classes by FP64 footprint (<= 2, 4, 8, 16, 32, 64, 128, 220 KB). Factorisation (eliminated tables):
  // the residual (rounded to an even row count) and the M x C table. Gram kernel (every table): the n = M - top residual
  // rows and the n bottom rows of the ce retained columns at an odd column stride.
  std::vector<int32_t> cls_tables[8], gram_tables[8];
  auto cls_of = [](int64_t b64) {
    int c = 0;
    while (c < 7 && b64 > (int64_t(2048) << c)) ++c;
    return c;
  };
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t M = d->table_nrows[t], C = d->table_ncols[t] - 1, top = d->table_top[t];
    if (t < neb) {
      // the warp's mbarrier, the residual and the table, each with room for a bulk copy's 16-byte alignment
      const int64_t rb = (8 * M + 32 + 15) & ~int64_t(15);
      int64_t b64 = 16 + rb + 8 * M * C + 32, b32 = 16 + rb + 4 * M * C + 32;
      if (b64 > QR_SMEM_LIMIT) throw Error(BLS_EUNSUPPORTED, "table " + std::to_string(t + 1) + " exceeds the shared-memory capacity of this build");
      // and the packed reflectors of the compact form, where they fit (the kernel checks the room it was given)
      if (d->e_dims[t] <= QR_WY_MAX && b64 + 8 * QR_WY_MAX * M <= QR_SMEM_LIMIT) {
        b64 += 8 * QR_WY_MAX * M;
        b32 += 4 * QR_WY_MAX * M;
      }
      const int c = cls_of(b64);
      cls_tables[c].push_back((int32_t)t);
      P->classes[c].bytes_f64 = std::max(P->classes[c].bytes_f64, b64);
      P->classes[c].bytes_f32 = std::max(P->classes[c].bytes_f32, b32);
      P->classes[c].maxc = std::max(P->classes[c].maxc, C);
    }
    // the warp's mbarrier, the residual rows and the retained columns: at stride M from one bulk copy (plus 32 bytes
    // of alignment room), or at the odd stride n | 1 from element copies; the larger of the two
    const int64_t n = M - top, ce = C - top, ns = n | 1;
    const int64_t cells = std::max<int64_t>(ce > 0 ? (ce - 1) * M + n : 0, ce * ns) + 8;
    const int64_t rb = (8 * n + 32 + 15) & ~int64_t(15);
    const int64_t g64 = 16 + rb + 8 * cells, g32 = 16 + rb + 4 * cells;
    if (g64 > QR_SMEM_LIMIT) throw Error(BLS_EUNSUPPORTED, "table " + std::to_string(t + 1) + " exceeds the shared-memory capacity of this build");
    const int c = cls_of(g64);
    gram_tables[c].push_back((int32_t)t);
    P->gram_classes[c].bytes_f64 = std::max(P->gram_classes[c].bytes_f64, g64);
    P->gram_classes[c].bytes_f32 = std::max(P->gram_classes[c].bytes_f32, g32);
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
  std::vector<int32_t> b_stride(nb);
  std::vector<int64_t> b_base(nb, 0), b_base_dense(nb);
  for (int64_t r2 = 0; r2 < nrb; ++r2)
    for (int64_t k = bcolptr[r2]; k < bcolptr[r2 + 1]; ++k) {
      b_stride[k] = (int32_t)col_h[r2];
      if (P->has_sparse) b_base[k] = Scolptr[boff_r[r2]] + brow_off[k];
      b_base_dense[k] = boff_r[browval[k]] + boff_r[r2] * nr;
    }
  // per table, its entry pairs (u2 outer, u1 <= u2 inner) and the S block (r1, r2) each adds to
  std::vector<int32_t> tp_ptr(nt + 1, 0), tp_blk;
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t u0 = d->table_ptr[t], kt = d->table_ptr[t + 1] - u0;
    for (int64_t b = 1; b < kt; ++b)
      if (d->entry_retained[u0 + b] <= d->entry_retained[u0 + b - 1]) throw Error(BLS_EINVAL, "table " + std::to_string(t + 1) + ": entries must be in ascending retained order");
    for (int64_t a2 = 0; a2 < kt; ++a2) {
      const int64_t r2 = d->entry_retained[u0 + a2], kb = bcolptr[r2], ke = bcolptr[r2 + 1];
      for (int64_t a1 = 0; a1 <= a2; ++a1) {
        const int64_t r1 = d->entry_retained[u0 + a1];
        const int64_t* f = std::lower_bound(browval.data() + kb, browval.data() + ke, r1);
        if (f == browval.data() + ke || *f != r1) throw Error(BLS_EPATTERN, "The sparse pattern has no block (" + std::to_string(r1 + 1) + ", " + std::to_string(r2 + 1) + ")");
        tp_blk.push_back((int32_t)(f - browval.data()));
      }
    }
    if (tp_blk.size() > (size_t)INT32_MAX) throw Error(BLS_EUNSUPPORTED, "too many entry pairs for this build");
    tp_ptr[t + 1] = (int32_t)tp_blk.size();
  }
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
    P->gram_classes[c].n = (int64_t)gram_tables[c].size();
    upload(P->gram_classes[c].tables, gram_tables[c], s);
  }
  upload(P->tp_ptr, tp_ptr, s);
  upload(P->tp_blk, tp_blk, s);
  {
    // SchurStructure's prefix-sum offsets (src/schur_structure.jl:70-166): eoffsets over d_e^2, coffsets over d_e d_r in
    // coupling order, which is the entry order of the eliminated tables (each point's entries in ascending retained order)
    std::vector<int64_t> eoff(neb), coff((size_t)d->table_ptr[neb]);
    int64_t eo = 0, co = 0;
    for (int64_t e = 0; e < neb; ++e) {
      eoff[e] = eo;
      eo += d->e_dims[e] * d->e_dims[e];
      for (int64_t u = d->table_ptr[e]; u < d->table_ptr[e + 1]; ++u) {
        coff[u] = co;
        co += d->e_dims[e] * d->r_dims[d->entry_retained[u]];
      }
    }
    P->E_len = eo;
    P->C_len = co;
    upload(P->t_eoff, eoff, s);
    upload(P->u_coff, coff, s);
    std::vector<int32_t> rptr(nrb + 1, 0), rent((size_t)nent), utab((size_t)nent);
    for (int64_t u = 0; u < nent; ++u) rptr[d->entry_retained[u] + 1] += 1;
    for (int64_t r = 0; r < nrb; ++r) rptr[r + 1] += rptr[r];
    std::vector<int32_t> fill(rptr.begin(), rptr.end() - 1);
    for (int64_t t = 0; t < nt; ++t)
      for (int64_t u = d->table_ptr[t]; u < d->table_ptr[t + 1]; ++u) {
        utab[u] = (int32_t)t;
        rent[fill[d->entry_retained[u]]++] = (int32_t)u;
      }
    upload(P->q_rptr, rptr, s);
    upload(P->q_rent, rent, s);
    upload(P->u_tab, utab, s);
    {   // each entry's column, retained offset, retained size and table in one 16-byte load (the products of the
        // reduced problem read them per entry)
      std::vector<int4> meta((size_t)nent);
      for (int64_t u = 0; u < nent; ++u) {
        const int64_t r = d->entry_retained[u];
        meta[(size_t)u] = make_int4((int)d->entry_col[u], (int)boff_r[r], (int)d->r_dims[r], utab[(size_t)u]);
      }
      upload(P->u_meta, meta, s);
    }
    // the reduced problem: build_reduced_jacobian_pattern's column heights (the reduced rows of every table coupled to
    // the column's retained block, tables in ascending order) and each entry's run position in those columns
    P->h_red.assign((size_t)nt + 1, 0);
    for (int64_t t = 0; t < nt; ++t) P->h_red[t + 1] = P->h_red[t] + d->table_nrows[t] - d->table_top[t];
    P->red_nrows = P->h_red[nt];
    {   // the table of every reduced row (reduced_mul!'s thread per row)
      std::vector<int32_t> rtab((size_t)P->red_nrows);
      for (int64_t t = 0; t < nt; ++t)
        for (int64_t i = P->h_red[t]; i < P->h_red[t + 1]; ++i) rtab[(size_t)i] = (int32_t)t;
      upload(P->red_tab, rtab, s);
    }
    P->h_jt_colptr.assign((size_t)nr + 1, 0);
    P->h_boff_r = boff_r;
    P->h_rdims.assign(d->r_dims, d->r_dims + nrb);
    P->h_rptr = rptr;
    P->h_rent_tab.resize((size_t)nent);
    std::vector<int64_t> runpos((size_t)nent, 0);
    for (int64_t r = 0; r < nrb; ++r) {
      int64_t h = 0;
      for (int32_t k = rptr[r]; k < rptr[r + 1]; ++k) {
        const int32_t u = rent[k], t = utab[u];
        P->h_rent_tab[k] = t;
        runpos[u] = h;
        h += d->table_nrows[t] - d->table_top[t];
      }
      for (int64_t j = 0; j < d->r_dims[r]; ++j) P->h_jt_colptr[boff_r[r] + j + 1] = P->h_jt_colptr[boff_r[r] + j] + h;
    }
    upload(P->t_red, P->h_red, s);
    upload(P->jt_colptr, P->h_jt_colptr, s);
    upload(P->u_runpos, runpos, s);
    P->q_total.alloc(sizeof(double));
  }
  upload(P->blk_stride, b_stride, s);
  upload(P->blk_base_sparse, b_base, s);
  upload(P->blk_base_dense, b_base_dense, s);
  P->status.alloc(4 * sizeof(long long));
  long long init[4] = {QNONE, QNONE, QNONE, QNONE};
  BLS_CUDA(cudaMemcpyAsync(P->status.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
  BLS_CUDA(cudaMallocHost(&P->host_status, 4 * sizeof(long long)));
  BLS_CUDA(cudaStreamSynchronize(s));
  return P.release();
}

// The verdict of the last reduce_qr (synchronises on the plan's stream)
static int qr_status(QRPlan* P, int64_t* failed_block) {
  cudaStream_t s = P->ctx->stream;
  BLS_CUDA(cudaMemcpyAsync(P->host_status, P->status.p, 3 * sizeof(long long), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  *failed_block = 0;
  if (P->host_status[2] != QNONE) throw Error(BLS_ECUDA, "a bulk copy of a table did not complete within its wait limit");
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
static int reduce_qr(QRPlan* P, T* F, double* Fr, const T* Rw, const double* Rr, const double* sc_e, double lambda, const double* sv,
                     int64_t* failed_block) {
  if (!(std::isfinite(lambda) && lambda >= 0)) throw Error(BLS_EINVAL, "lambda must be finite and non-negative, got " + std::to_string(lambda));
  cudaStream_t s = P->ctx->stream;
  long long* st = P->status.as<long long>();
  k_qr_begin<<<1, 1, 0, s>>>(st);
  k_qr_check<<<grid_for(P->ne, 256), 256, 0, s>>>(sc_e, P->ne, st);
  P->launches += 2;
  // bulk copies need the buffers' starts on 16-byte boundaries (the device allocators give 256); otherwise the tables
  // are staged element by element
  const bool bulk = P->bulk && (reinterpret_cast<uintptr_t>(Rw) & 15) == 0 && (reinterpret_cast<uintptr_t>(Rr) & 15) == 0;
  // the factored tables go out by bulk copies too when F keeps the raw tables' 16-byte offsets
  const int bulk_mode = bulk ? 1 | ((reinterpret_cast<uintptr_t>(F) & 15) == 0 ? 2 : 0) : 0;
  fork_sides(P, s);
  for (int c = 0, q = 0; c < 8; ++c) {
    const auto& k = P->classes[c];
    if (k.n == 0) continue;
    cudaStream_t cs = class_stream(P, s, q++);
    const int64_t wb = ((std::is_same<T, double>::value ? k.bytes_f64 : k.bytes_f32) + 15) & ~int64_t(15);
    // lanes per table from the widest table of the class: a lane per column in the reflector updates
    int G = k.maxc <= 24 ? 8 : k.maxc <= 48 ? 16 : 32;
    const void* kg = G == 8 ? reinterpret_cast<const void*>(k_qr_tables<T, 8>) : G == 16 ? reinterpret_cast<const void*>(k_qr_tables<T, 16>)
                                                                                          : reinterpret_cast<const void*>(k_qr_tables<T, 32>);
    int tpc = tables_per_cta(wb, G, warp_cap(kg));
    if (tpc == 0) {
      G = 32;
      tpc = warps_per_cta(wb);
    }
    const size_t smem = (size_t)(wb * tpc);
    auto launch = [&](auto kern) {
      set_smem(reinterpret_cast<const void*>(kern), smem);
      kern<<<(unsigned)((k.n + tpc - 1) / tpc), tpc * G, smem, cs>>>(
          k.n, (int)wb, k.tables.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(),
          P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(), P->boff_r.as<int32_t>(), P->r_dims.as<int32_t>(),
          P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(), (int)P->nr, Rw, Rr, sc_e, lambda, sv, F, Fr, Rw + P->raw_len, Rr + P->res_len,
          bulk_mode, st);
    };
    if (G == 8) launch(k_qr_tables<T, 8>);
    else if (G == 16) launch(k_qr_tables<T, 16>);
    else launch(k_qr_tables<T, 32>);
    P->launches += 1;
  }
  join_sides(P, s);
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
  return qr_status(P, failed_block);
}

// One launch per Gram class: MODE 0 writes S (sparse or dense) and g, MODE 1 the diagonal blocks D.
template <class T, int MODE>
static void gram(QRPlan* P, T* S, bool dense, double* g, const T* F, const double* Fr, bool from_raw = false) {
  cudaStream_t s = P->ctx->stream;
  const bool bulk = P->bulk && (reinterpret_cast<uintptr_t>(F) & 15) == 0 && (reinterpret_cast<uintptr_t>(Fr) & 15) == 0;
  fork_sides(P, s);
  for (int c = 0, q = 0; c < 8; ++c) {
    const auto& k = P->gram_classes[c];
    if (k.n == 0) continue;
    cudaStream_t cs = class_stream(P, s, q++);
    const int64_t wb = ((std::is_same<T, double>::value ? k.bytes_f64 : k.bytes_f32) + 15) & ~int64_t(15);
    auto kern = P->all6 ? k_qr_gram<T, MODE, true> : k_qr_gram<T, MODE, false>;
    const int wpc = std::max(1, tables_per_cta(wb, 32, warp_cap(reinterpret_cast<const void*>(kern))));
    const size_t smem = (size_t)(wb * wpc);
    set_smem(reinterpret_cast<const void*>(kern), smem);
    kern<<<(unsigned)((k.n + wpc - 1) / wpc), 32 * wpc, smem, cs>>>(
        k.n, (int)wb, k.tables.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(),
        P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_ret.as<int32_t>(), P->u_col.as<int32_t>(), P->r_dims.as<int32_t>(),
        P->boff_r.as<int32_t>(), P->tp_ptr.as<int32_t>(), P->tp_blk.as<int32_t>(),
        dense ? P->blk_base_dense.as<int64_t>() : P->blk_base_sparse.as<int64_t>(), dense ? nullptr : P->blk_stride.as<int32_t>(), P->nr,
        P->doff.as<int64_t>(), P->max_dr, F, Fr, S, g, from_raw ? 1 : 0, F + P->raw_len, Fr + P->res_len, bulk ? 1 : 0,
        P->status.as<long long>());
    P->launches += 1;
  }
  join_sides(P, s);
  BLS_CUDA(cudaGetLastError());
}

template <class T>
static void normal(QRPlan* P, T* S, bool dense, double* g, const T* F, const double* Fr) {
  if (!dense && !P->has_sparse) throw Error(BLS_EINVAL, "the QR plan was created without a sparse pattern");
  cudaStream_t s = P->ctx->stream;
  const int64_t nS = dense ? P->nr * P->nr : P->nnzS;
  k_fill_t<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(nS, 256), 148 * 8)), 256, 0, s>>>(S, nS);
  k_fill_t<double><<<(unsigned)std::max(1, grid_for(P->nr, 256)), 256, 0, s>>>(g, P->nr);
  P->launches += 2;
  gram<T, 0>(P, S, dense, g, F, Fr);
}

// H = J'J and b = J'r from the raw tables into the SchurBlockHessian layout of the same structure: E_data, C_data,
// R on the reduced pattern (upper blocks; sparse S.nzval layout or dense column-major nr x nr) and b = [b_r; b_e].
template <class T>
static void assemble(QRPlan* P, const T* J, const double* r, T* E, T* Cd, T* R, bool dense, double* b) {
  if (!dense && !P->has_sparse) throw Error(BLS_EINVAL, "the QR plan was created without a sparse pattern");
  if (!J || !r || !E || !Cd || !R || !b) throw Error(BLS_EINVAL, "a device pointer is NULL");
  cudaStream_t s = P->ctx->stream;
  const int64_t nS = dense ? P->nr * P->nr : P->nnzS;
  k_fill_t<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(nS, 256), 148 * 8)), 256, 0, s>>>(R, nS);
  k_fill_t<double><<<(unsigned)std::max(1, grid_for(P->nr, 256)), 256, 0, s>>>(b, P->nr);
  k_qr_point_gram<T><<<(unsigned)grid_for(P->neblocks * 32, 128), 128, 0, s>>>(
      P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(),
      P->u_ret.as<int32_t>(), P->u_col.as<int32_t>(), P->r_dims.as<int32_t>(), P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(),
      P->t_eoff.as<int64_t>(), P->u_coff.as<int64_t>(), J, r, E, Cd, b + P->nr);
  P->launches += 3;
  gram<T, 0>(P, R, dense, b, J, r, true);
}

// jtr! (MODE 0) / jtj_diag! (MODE 1) of the tables D with residual Rv into out[nr + ne]
template <class T, int MODE>
static void jt_columns(QRPlan* P, double* out, const T* D, const double* Rv) {
  if (!out || !D || (MODE == 0 && !Rv)) throw Error(BLS_EINVAL, "a device pointer is NULL");
  cudaStream_t s = P->ctx->stream;
  k_jt_retained<T, MODE><<<(unsigned)grid_for(P->nrblocks * 32, 256), 256, 0, s>>>(
      P->nrblocks, P->q_rptr.as<int32_t>(), P->q_rent.as<int32_t>(), P->u_tab.as<int32_t>(), P->u_col.as<int32_t>(), P->r_dims.as<int32_t>(),
      P->boff_r.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), D, Rv, out);
  k_jt_eliminated<T, MODE><<<(unsigned)grid_for(P->neblocks, 128), 128, 0, s>>>(
      P->neblocks, P->nr, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(),
      P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(), D, Rv, out);
  P->launches += 2;
  BLS_CUDA(cudaGetLastError());
}

template <class T>
static double jtj_quadform(QRPlan* P, const T* D, const double* v) {
  if (!D || !v) throw Error(BLS_EINVAL, "a device pointer is NULL");
  cudaStream_t s = P->ctx->stream;
  double* tot = P->q_total.as<double>();
  k_fill_t<double><<<1, 32, 0, s>>>(tot, 1);
  k_jtj_quadform<T><<<(unsigned)grid_for(P->ntables * 32, 256), 256, 0, s>>>(
      P->ntables, P->neblocks, P->nr, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(), P->t_ptr.as<int32_t>(),
      P->u_ret.as<int32_t>(), P->u_col.as<int32_t>(), P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), P->e_dims.as<int32_t>(),
      P->boff_e.as<int32_t>(), D, v, tot);
  P->launches += 2;
  double h = 0.0;
  BLS_CUDA(cudaMemcpyAsync(&h, tot, sizeof(double), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  return h;
}

template <class T>
static void diagonal_blocks(QRPlan* P, T* D, const T* F) {
  cudaStream_t s = P->ctx->stream;
  const int64_t nD = P->ndiag;
  k_fill_t<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(nD, 256), 148 * 8)), 256, 0, s>>>(D, nD);
  P->launches += 1;
  gram<T, 1>(P, D, false, nullptr, F, nullptr);
}

// ---- LSMR on the reduced problem (ext/KrylovExt.jl:25-132): min || A x - [r~; 0] ||, A = [J~; diag(sqrt(lambda s_r))]
// (reduced_nrows + nr rows), with the block-Jacobi N = D^-1, D the diagonal blocks of A'A = J~'J~ + lambda diag(s_r).
// Krylov's N-preconditioned LSMR is ordinary LSMR on B = A C with C C' = N; with D = L L' that is C = L^-T, so the
// Golub-Kahan vectors u, v are B's, while h, hbar and x are kept in the original variables (t = L^-T v is what both B v
// and the h update need). The vectors are FP64 on the device; the scalar recurrences of Fong & Saunders (SIAM J. Sci.
// Comput. 33 (2011), LSMR with its estimates of ||r||, ||A'r||, ||A|| and cond(A)) run on the host.

// The diagonal blocks of J~'J~ in FP64, straight from the factored tables, in two passes as reduced_tmul!: a thread
// per (entry, column pair a <= b) forms the pair's dot product over the entry's reduced rows into
// part[u * npair + b (b + 1) / 2 + a]; a warp per (retained block, pair) sums its entries in order into both triangles
// of L's block (column-major, at doff).
template <class T>
__global__ void __launch_bounds__(256) k_lsmr_diag_entries(int64_t nent, int npair, const int4* __restrict__ meta,
                                                           const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_top,
                                                           const int64_t* __restrict__ t_raw, const T* __restrict__ F,
                                                           double* __restrict__ part) {
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= nent * npair) return;
  const int64_t u = gid / npair;
  const int p = (int)(gid - u * npair);
  int b = (int)((sqrtf(8.0f * p + 1.0f) - 1.0f) * 0.5f);
  while ((b + 1) * (b + 2) / 2 <= p) ++b;
  while (b * (b + 1) / 2 > p) --b;
  const int a = p - b * (b + 1) / 2;
  const int4 q = meta[u];   // column, retained offset, retained size, table
  if (b >= q.z) return;
  const int t = q.w, M = t_rows[t], top = t_top[t], n = M - top;
  const T* ca = F + t_raw[t] + (int64_t)(q.x + a) * M + top;
  const T* cb = F + t_raw[t] + (int64_t)(q.x + b) * M + top;
  double acc = 0.0;
#pragma unroll 4
  for (int i = 0; i < n; ++i) acc += (double)ca[i] * (double)cb[i];
  part[gid] = acc;
}

__global__ void __launch_bounds__(256) k_lsmr_diag_reduce(int64_t nrb, int npair, const int32_t* __restrict__ rptr,
                                                          const int32_t* __restrict__ rent, const int32_t* __restrict__ r_dims,
                                                          const int64_t* __restrict__ doff, const double* __restrict__ part,
                                                          double* __restrict__ L) {
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t r = gw / npair;
  const int p = (int)(gw - r * npair);
  if (r >= nrb) return;
  int b = 0;
  while ((b + 1) * (b + 2) / 2 <= p) ++b;
  const int a = p - b * (b + 1) / 2, d = r_dims[r];
  if (b >= d) return;   // uniform across the warp
  double acc = 0.0;
  for (int k = rptr[r] + lane; k < rptr[r + 1]; k += 32) acc += part[(int64_t)rent[k] * npair + p];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    L[doff[r] + a + (int64_t)d * b] = acc;
    L[doff[r] + b + (int64_t)d * a] = acc;
  }
}

// D_b + sqd^2 on its diagonal, then its Cholesky factor (lower, column-major) in place in L; a thread per block. A
// block that is not positive definite (or not finite) records the lowest such block in *bad.
__global__ void k_lsmr_factor(int64_t nrb, const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                              const int64_t* __restrict__ doff, const double* __restrict__ sqd, double* __restrict__ L,
                              int* __restrict__ bad) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nrb) return;
  const int d = r_dims[b], ro = boff_r[b];
  double* a = L + doff[b];
  for (int i = 0; i < d; ++i) a[i + d * i] += sqd[ro + i] * sqd[ro + i];
  for (int j = 0; j < d; ++j) {
    double p = a[j + d * j];
    for (int k = 0; k < j; ++k) p -= a[j + d * k] * a[j + d * k];
    if (!(p > 0.0) || !isfinite(p)) {
      atomicMin(bad, (int)b);
      return;
    }
    const double ljj = sqrt(p);
    a[j + d * j] = ljj;
    for (int i = j + 1; i < d; ++i) {
      double q = a[i + d * j];
      for (int k = 0; k < j; ++k) q -= a[i + d * k] * a[j + d * k];
      a[i + d * j] = q / ljj;
    }
  }
}

__device__ __forceinline__ void warp_sum_add(double v, double* out) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out, v);
}

// v = L^-1 (sc (w + sqd .* ub)) + gamma v, block by block (w is overwritten), and acc += |v|^2; a thread per block.
// This is B' u - beta v with u = sc ub_raw: w = J~' u_top(raw), ub = the raw bottom of u.
__global__ void k_lsmr_fwd(int64_t nrb, const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                           const int64_t* __restrict__ doff, const double* __restrict__ L, double* __restrict__ w,
                           const double* __restrict__ sqd, const double* __restrict__ ub, double sc, double gamma,
                           double* __restrict__ v, double* __restrict__ acc) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double nn = 0.0;
  if (b < nrb) {
    const int d = r_dims[b], ro = boff_r[b];
    const double* a = L + doff[b];
    for (int i = 0; i < d; ++i) {
      double q = sc * (w[ro + i] + sqd[ro + i] * ub[ro + i]);
      for (int k = 0; k < i; ++k) q -= a[i + d * k] * w[ro + k];
      w[ro + i] = q / a[i + d * i];
    }
    for (int i = 0; i < d; ++i) {
      const double z = w[ro + i] + gamma * v[ro + i];
      v[ro + i] = z;
      nn += z * z;
    }
  }
  warp_sum_add(nn, acc);
}

// v *= sc, then t = L^-T v, block by block; a thread per block
__global__ void k_lsmr_bwd(int64_t nrb, const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                           const int64_t* __restrict__ doff, const double* __restrict__ L, double sc, double* __restrict__ v,
                           double* __restrict__ t) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nrb) return;
  const int d = r_dims[b], ro = boff_r[b];
  const double* a = L + doff[b];
  for (int i = 0; i < d; ++i) v[ro + i] *= sc;
  for (int i = d - 1; i >= 0; --i) {
    double q = v[ro + i];
    for (int k = i + 1; k < d; ++k) q -= a[k + d * i] * t[ro + k];
    t[ro + i] = q / a[i + d * i];
  }
}

// u = B t - a u with B t = [J~ t; sqd .* t] (a thread per row of u: a reduced row's product as reduced_mul! forms it,
// then the damping rows), acc += |u|^2
template <class T>
__global__ void __launch_bounds__(256) k_lsmr_bv(int64_t mt, int64_t nr, const int32_t* __restrict__ red_tab,
                                                 const int32_t* __restrict__ t_rows, const int32_t* __restrict__ t_top,
                                                 const int64_t* __restrict__ t_raw, const int64_t* __restrict__ t_red,
                                                 const int32_t* __restrict__ t_ptr, const int4* __restrict__ meta,
                                                 const T* __restrict__ F, const double* __restrict__ sqd,
                                                 const double* __restrict__ t, double a,
                                                 double* __restrict__ u, double* __restrict__ acc) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double nn = 0.0;
  if (row < mt) {
    const int tb = red_tab[row];
    const int M = t_rows[tb], top = t_top[tb];
    const int64_t raw = t_raw[tb] + top + (row - t_red[tb]);
    double y = 0.0;
    for (int e = t_ptr[tb]; e < t_ptr[tb + 1]; ++e) {
      const int4 q = meta[e];   // column, retained offset, retained size
      const T* col = F + raw + (int64_t)q.x * M;
      if (q.z == 6) {           // the common camera block: six independent loads in flight
        T f[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) f[j] = col[(int64_t)j * M];
#pragma unroll
        for (int j = 0; j < 6; ++j) y += (double)f[j] * t[q.y + j];
      } else {
        for (int j = 0; j < q.z; ++j) y += (double)col[(int64_t)j * M] * t[q.y + j];
      }
    }
    const double z = y - a * u[row];
    u[row] = z;
    nn = z * z;
  } else if (row < mt + nr) {
    const double z = sqd[row - mt] * t[row - mt] - a * u[row];
    u[row] = z;
    nn = z * z;
  }
  warp_sum_add(nn, acc);
}

// One iteration's end, a thread per block: v *= sc, t = L^-T v, then for the block's entries hbar = h - c1 hbar,
// x += c2 hbar, h = t - c3 h; acc += |x|^2
__global__ void k_lsmr_bwd_update(int64_t nrb, const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boff_r,
                                  const int64_t* __restrict__ doff, const double* __restrict__ L, double sc, double* __restrict__ v,
                                  double* __restrict__ t, double* __restrict__ h, double* __restrict__ hbar, double* __restrict__ x,
                                  double c1, double c2, double c3, double* __restrict__ acc) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double nn = 0.0;
  if (b < nrb) {
    const int d = r_dims[b], ro = boff_r[b];
    const double* a = L + doff[b];
    for (int i = 0; i < d; ++i) v[ro + i] *= sc;
    for (int i = d - 1; i >= 0; --i) {
      double q = v[ro + i];
      for (int k = i + 1; k < d; ++k) q -= a[k + d * i] * t[ro + k];
      t[ro + i] = q / a[i + d * i];
    }
    for (int i = ro; i < ro + d; ++i) {
      const double hb = h[i] - c1 * hbar[i];
      hbar[i] = hb;
      const double xi = x[i] + c2 * hb;
      x[i] = xi;
      h[i] = t[i] - c3 * h[i];
      nn += xi * xi;
    }
  }
  warp_sum_add(nn, acc);
}

// sqd = sqrt(lambda s_r) (s_r NULL: sqrt(lambda)); u's bottom rows zero; acc[0] += |r~|^2 (u's top, already written)
__global__ void k_lsmr_init(int64_t mt, int64_t nr, double lambda, const double* __restrict__ s_r, double* __restrict__ sqd,
                            double* __restrict__ u, double* __restrict__ acc) {
  double nn = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < mt + nr; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < mt) {
      nn += u[i] * u[i];
    } else {
      sqd[i - mt] = sqrt(lambda * (s_r ? s_r[i - mt] : 1.0));
      u[i] = 0.0;
    }
  }
  warp_sum_add(nn, acc);
}

struct LsmrOut {
  int64_t iterations = 0;
  int istop = 0;
  double normr = 0, normar = 0, normA = 0, condA = 0, normx = 0;
};

// The stopping tests' order and meaning (Fong & Saunders): 1 ||r|| small (a compatible system), 2 ||A'r|| small (a
// least-squares solution), 3 cond(A) above conlim, 4-6 the same at machine precision, 7 itmax iterations.
template <class T>
static int lsmr_reduced(QRPlan* P, const T* F, const double* Fr, double lambda, const double* s_r, double* x, double atol,
                        double btol, double conlim, int64_t itmax, LsmrOut* out) {
  cudaStream_t s = P->ctx->stream;
  const int64_t mt = P->red_nrows, nr = P->nr, nrb = P->nrblocks, m = mt + nr;
  if (!P->ls_u.p) {
    P->ls_u.alloc(sizeof(double) * (size_t)std::max<int64_t>(m, 1));
    for (DevBuf* b : {&P->ls_v, &P->ls_h, &P->ls_hbar, &P->ls_t, &P->ls_w, &P->ls_sqd})
      b->alloc(sizeof(double) * (size_t)std::max<int64_t>(nr, 1));
    P->ls_L.alloc(sizeof(double) * (size_t)std::max<int64_t>(P->ndiag, 1));
    P->ls_acc.alloc(sizeof(double) * 4);
    P->ls_flag.alloc(sizeof(int));
    BLS_CUDA(cudaMallocHost(reinterpret_cast<void**>(&P->ls_host), sizeof(double) * 4));
  }
  double *u = P->ls_u.as<double>(), *v = P->ls_v.as<double>(), *h = P->ls_h.as<double>();
  double *hbar = P->ls_hbar.as<double>(), *t = P->ls_t.as<double>(), *w = P->ls_w.as<double>(), *sqd = P->ls_sqd.as<double>();
  double *L = P->ls_L.as<double>(), *acc = P->ls_acc.as<double>(), *hv = P->ls_host;
  int* flag = P->ls_flag.as<int>();
  const int32_t *rd = P->r_dims.as<int32_t>(), *bo = P->boff_r.as<int32_t>();
  const int64_t* doff = P->doff.as<int64_t>();
  const unsigned gm = (unsigned)std::max(1, std::min(grid_for(m, 256), 148 * 8));
  const unsigned gb = (unsigned)std::max(1, grid_for(nrb, 128));
  auto read = [&](int k) {   // the first k norm accumulators to the host
    BLS_CUDA(cudaMemcpyAsync(hv, acc, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
  };
  *out = LsmrOut();
  // u = [r~; 0], sqd = sqrt(lambda s_r), |r~|^2; D + lambda s_r factored; x = 0
  BLS_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 4, s));
  BLS_CUDA(cudaMemsetAsync(flag, 0x7f, sizeof(int), s));
  BLS_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)nr, s));
  if (mt > 0)
    k_reduced_residual<<<(unsigned)std::max(1, grid_for(P->ntables * 32, 256)), 256, 0, s>>>(
        P->ntables, P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_res.as<int64_t>(), P->t_red.as<int64_t>(), Fr, u);
  k_lsmr_init<<<gm, 256, 0, s>>>(mt, nr, lambda, s_r, sqd, u, acc);
  {
    if (P->rdmax == 0)
      for (int64_t d : P->h_rdims) P->rdmax = std::max<int>(P->rdmax, (int)d);
    const int np = std::max(P->rdmax, 1) * (std::max(P->rdmax, 1) + 1) / 2;
    const size_t need = sizeof(double) * (size_t)std::max<int64_t>(P->nentries * np, 1);
    if (P->ls_part.bytes < need) P->ls_part.alloc(need);
    BLS_CUDA(cudaMemsetAsync(L, 0, sizeof(double) * (size_t)P->ndiag, s));   // blocks without entries stay zero
    if (P->nentries > 0)
      k_lsmr_diag_entries<T><<<(unsigned)grid_for(P->nentries * np, 256), 256, 0, s>>>(
          P->nentries, np, P->u_meta.as<int4>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(), F,
          P->ls_part.as<double>());
    k_lsmr_diag_reduce<<<(unsigned)std::max(1, grid_for(nrb * np * 32, 256)), 256, 0, s>>>(
        nrb, np, P->q_rptr.as<int32_t>(), P->q_rent.as<int32_t>(), rd, doff, P->ls_part.as<double>(), L);
  }
  k_lsmr_factor<<<gb, 128, 0, s>>>(nrb, rd, bo, doff, sqd, L, flag);
  P->launches += 4 + (mt > 0);
  BLS_CUDA(cudaGetLastError());
  BLS_CUDA(cudaMemcpyAsync(hv, acc, sizeof(double), cudaMemcpyDeviceToHost, s));
  int bad = 0;
  BLS_CUDA(cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  const double bb = hv[0];
  if (!std::isfinite(bb)) return BLS_NOT_PD;          // a non-finite reduced residual
  if (lambda == 0 && mt < nr) return BLS_NOT_PD;      // undamped with fewer reduced rows than variables: rank deficient
  if (bad != 0x7f7f7f7f) return BLS_NOT_PD;           // a diagonal block of A'A is not positive definite
  double beta = std::sqrt(bb);
  out->normr = beta;
  if (nr == 0 || beta == 0) return BLS_OK;            // x = 0 solves it
  // alpha v = B' u with u = u_raw / beta; t = L^-T v; h = t
  BLS_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 4, s));
  BLS_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * (size_t)nr, s));
  BLS_CUDA(cudaMemsetAsync(hbar, 0, sizeof(double) * (size_t)nr, s));
  launch_reduced_tmul<T>(P, F, u, w);
  k_lsmr_fwd<<<gb, 128, 0, s>>>(nrb, rd, bo, doff, L, w, sqd, u + mt, 1.0 / beta, 0.0, v, acc + 1);
  P->launches += 1;
  read(2);
  double alpha = std::sqrt(hv[1]);
  k_lsmr_bwd<<<gb, 128, 0, s>>>(nrb, rd, bo, doff, L, alpha > 0 ? 1.0 / alpha : 1.0, v, t);
  P->launches += 1;
  BLS_CUDA(cudaMemcpyAsync(h, t, sizeof(double) * (size_t)nr, cudaMemcpyDeviceToDevice, s));
  double uscale = 1.0 / beta;   // u = uscale * u_raw

  double zetabar = alpha * beta, alphabar = alpha, rho = 1, rhobar = 1, cbar = 1, sbar = 0;
  double betadd = beta, betad = 0, rhodold = 1, tautildeold = 0, thetatilde = 0, zeta = 0, dsum = 0;
  double normA2 = alpha * alpha, maxrbar = 0, minrbar = 1e100, normA = std::sqrt(normA2), condA = 1;
  const double normb = beta, ctol = conlim > 0 ? 1.0 / conlim : 0.0;
  double normr = beta, normar = alpha * beta, normx = 0;
  int64_t itn = 0;
  int istop = 0;
  if (normar == 0) {
    out->normr = normr;
    return BLS_OK;
  }
  if (itmax == 0) {   // no iteration allowed: x = 0, stopped on itmax
    out->istop = 7;
    out->normr = normr;
    out->normar = normar;
    BLS_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)nr, s));
    return BLS_NOT_CONVERGED;
  }
  // The tests of an iteration need ||x||, which the update kernel accumulates; they are evaluated at the next
  // iteration's first read-back, after B v of the next step has been launched (at itmax, without it)
  auto tests = [&]() -> int {
    const double test1 = normr / normb;
    const double t2d = normA * normr;
    const double test2 = t2d != 0 ? normar / t2d : INFINITY;
    const double test3 = 1.0 / condA;
    const double t1 = test1 / (1.0 + normA * normx / normb);
    const double rtol = btol + atol * normA * normx / normb;
    int k = 0;
    if (itn >= itmax) k = 7;
    if (1.0 + test3 <= 1.0) k = 6;
    if (1.0 + test2 <= 1.0) k = 5;
    if (1.0 + t1 <= 1.0) k = 4;
    if (test3 <= ctol) k = 3;
    if (test2 <= atol) k = 2;
    if (test1 <= rtol) k = 1;
    return k;
  };
  bool pending = false;
  for (;;) {
    // u_raw = B v - alpha u
    if (itn < itmax) {
      BLS_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 2, s));
      k_lsmr_bv<T><<<(unsigned)grid_for(m, 256), 256, 0, s>>>(
          mt, nr, P->red_tab.as<int32_t>(), P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_raw.as<int64_t>(),
          P->t_red.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_meta.as<int4>(), F, sqd, t, alpha * uscale, u, acc);
      P->launches += 1;
    }
    read(3);
    if (pending) {
      normx = std::sqrt(hv[2]);
      istop = tests();
      if (istop) break;
    }
    ++itn;
    beta = std::sqrt(hv[0]);
    if (!std::isfinite(beta)) return BLS_NOT_PD;
    if (beta > 0) {
      uscale = 1.0 / beta;
      // v_raw = B' u - beta v, alpha = |v_raw|, v = v_raw / alpha, t = L^-T v
      launch_reduced_tmul<T>(P, F, u, w);
      k_lsmr_fwd<<<gb, 128, 0, s>>>(nrb, rd, bo, doff, L, w, sqd, u + mt, uscale, -beta, v, acc + 1);
      P->launches += 1;
      read(2);
      alpha = std::sqrt(hv[1]);
      if (!std::isfinite(alpha)) return BLS_NOT_PD;
    } else {
      uscale = 0.0;
    }
    const double vscale = beta > 0 && alpha > 0 ? 1.0 / alpha : 1.0;   // v unchanged when beta = 0: t is recomputed as is
    // the plane rotations (no regularisation in LSMR itself: the damping rows are part of A)
    const double alphahat = alphabar;
    const double rhoold = rho;
    rho = std::hypot(alphahat, beta);
    const double c = alphahat / rho, sn = beta / rho;
    const double thetanew = sn * alpha;
    alphabar = c * alpha;
    const double rhobarold = rhobar, zetaold = zeta, thetabar = sbar * rho, rhotemp = cbar * rho;
    rhobar = std::hypot(cbar * rho, thetanew);
    cbar = cbar * rho / rhobar;
    sbar = thetanew / rhobar;
    zeta = cbar * zetabar;
    zetabar = -sbar * zetabar;
    // hbar = h - (thetabar rho / (rhoold rhobarold)) hbar; x += (zeta / (rho rhobar)) hbar; h = t - (thetanew / rho) h
    BLS_CUDA(cudaMemsetAsync(acc + 2, 0, sizeof(double), s));
    k_lsmr_bwd_update<<<gb, 128, 0, s>>>(nrb, rd, bo, doff, L, vscale, v, t, h, hbar, x, thetabar * rho / (rhoold * rhobarold),
                                         zeta / (rho * rhobar), thetanew / rho, acc + 2);
    P->launches += 1;
    // ||r||: the rotations applied to (betadd, betad) and the running tau
    const double betaacute = betadd, betahat = c * betaacute;
    betadd = -sn * betaacute;
    const double thetatildeold = thetatilde, rhotildeold = std::hypot(rhodold, thetabar);
    const double ctildeold = rhodold / rhotildeold, stildeold = thetabar / rhotildeold;
    thetatilde = stildeold * rhobar;
    rhodold = ctildeold * rhobar;
    betad = -stildeold * betad + ctildeold * betahat;
    tautildeold = (zetaold - thetatildeold * tautildeold) / rhotildeold;
    const double taud = (zeta - thetatilde * tautildeold) / rhodold;
    normr = std::sqrt(dsum + (betad - taud) * (betad - taud) + betadd * betadd);
    // ||A|| (of B) and cond(A)
    normA2 += beta * beta;
    normA = std::sqrt(normA2);
    normA2 += alpha * alpha;
    maxrbar = std::max(maxrbar, rhobarold);
    if (itn > 1) minrbar = std::min(minrbar, rhobarold);
    condA = std::max(maxrbar, rhotemp) / std::min(minrbar, rhotemp);
    normar = std::fabs(zetabar);
    pending = true;
  }
  out->iterations = itn;
  out->istop = istop;
  out->normr = normr;
  out->normar = normar;
  out->normA = normA;
  out->condA = condA;
  out->normx = normx;
  if (!std::isfinite(normx)) return BLS_NOT_PD;
  if (istop == 7) return BLS_NOT_CONVERGED;
  if (istop == 3 || istop == 6) return BLS_NOT_PD;   // cond(A) above conlim: not solved
  return BLS_OK;
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

int bls_qr_normal_residual(bls_qr_plan* P, int dtype, const void* J, const double* r, const double* scaling, double lambda,
                           const double* x, double* y, double* d) {
  QR_GUARD({
    if (!P || !J || !r || !scaling || !x || !y || !d) throw Error(BLS_EINVAL, "a device pointer is NULL");
    if (!(std::isfinite(lambda) && lambda >= 0)) throw Error(BLS_EINVAL, "lambda must be finite and non-negative");
    cudaStream_t s = P->ctx->stream;
    const unsigned grid = (unsigned)std::max<int64_t>(1, grid_for(P->ntables * 32, 256));
    if (dtype == BLS_F64) {
      k_qr_rows_residual<double><<<grid, 256, 0, s>>>(P->ntables, P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(),
                                                     P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(),
                                                     P->u_ret.as<int32_t>(), P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(),
                                                     P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(), P->nr, (const double*)J, r, x, y);
      jt_columns<double, 0>(P, d, (const double*)J, y);
    } else if (dtype == BLS_F32) {
      k_qr_rows_residual<float><<<grid, 256, 0, s>>>(P->ntables, P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(),
                                                    P->t_raw.as<int64_t>(), P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(),
                                                    P->u_ret.as<int32_t>(), P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(),
                                                    P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(), P->nr, (const float*)J, r, x, y);
      jt_columns<float, 0>(P, d, (const float*)J, y);
    } else {
      throw Error(BLS_EINVAL, "unknown dtype");
    }
    const int64_t n = P->nr + P->ne;
    k_sub_damping<<<(unsigned)std::max<int64_t>(1, grid_for(n, 256)), 256, 0, s>>>(n, lambda, scaling, x, d);
    P->launches += 2;
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_qr_reduce_rhs(bls_qr_plan* P, int dtype, const void* F, const double* d, double* w, double* d_r) {
  QR_GUARD({
    if (!P || !F || !d || !w || !d_r) throw Error(BLS_EINVAL, "a device pointer is NULL");
    if (P->max_de > 16) throw Error(BLS_EUNSUPPORTED, "eliminated blocks above 16 variables");
    cudaStream_t s = P->ctx->stream;
    BLS_CUDA(cudaMemcpyAsync(d_r, d, sizeof(double) * P->nr, cudaMemcpyDeviceToDevice, s));
    const unsigned grid = (unsigned)std::max<int64_t>(1, grid_for(P->neblocks, 128));
    if (dtype == BLS_F64)
      k_qr_reduce_rhs<double><<<grid, 128, 0, s>>>(P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(),
                                                  P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(), P->r_dims.as<int32_t>(),
                                                  P->boff_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(), P->nr,
                                                  (const double*)F, d, w, d_r);
    else if (dtype == BLS_F32)
      k_qr_reduce_rhs<float><<<grid, 128, 0, s>>>(P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(),
                                                 P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(), P->r_dims.as<int32_t>(),
                                                 P->boff_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(), P->nr,
                                                 (const float*)F, d, w, d_r);
    else
      throw Error(BLS_EINVAL, "unknown dtype");
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_qr_backsubstitute_rhs(bls_qr_plan* P, int dtype, const void* F, const double* w, const double* x_r, double* x_e) {
  QR_GUARD({
    if (!P || !F || !w || !x_r || !x_e) throw Error(BLS_EINVAL, "a device pointer is NULL");
    cudaStream_t s = P->ctx->stream;
    const unsigned grid = (unsigned)std::max<int64_t>(1, grid_for(P->neblocks, 128));
    if (dtype == BLS_F64)
      k_qr_backsub<double><<<grid, 128, 0, s>>>(P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(),
                                               P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(),
                                               P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(),
                                               (const double*)F, nullptr, x_r, x_e, w);
    else if (dtype == BLS_F32)
      k_qr_backsub<float><<<grid, 128, 0, s>>>(P->neblocks, P->t_rows.as<int32_t>(), P->t_cols.as<int32_t>(), P->t_raw.as<int64_t>(),
                                              P->t_res.as<int64_t>(), P->t_ptr.as<int32_t>(), P->u_col.as<int32_t>(), P->u_ret.as<int32_t>(),
                                              P->r_dims.as<int32_t>(), P->boff_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boff_e.as<int32_t>(),
                                              (const float*)F, nullptr, x_r, x_e, w);
    else
      throw Error(BLS_EINVAL, "unknown dtype");
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_qr_plan_set_staging(bls_qr_plan* plan, int bulk) {
  if (!plan) return BLS_EINVAL;
  static_cast<QRPlan*>(plan)->bulk = bulk != 0;
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

int bls_qr_query_status(bls_qr_plan* P, int64_t* failed_block) {
  QR_GUARD({
    if (!P || !failed_block) throw Error(BLS_EINVAL, "null argument");
    return qr_status(P, failed_block);
  })
}

int64_t bls_qr_plan_counters(bls_qr_plan* P) {
  if (!P) return -1;
  const int64_t n = P->launches;
  P->launches = 0;
  return n;
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

int bls_jtr(bls_qr_plan* P, int dtype, double* g, const void* D, const double* Rv) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (dtype == BLS_F64) jt_columns<double, 0>(P, g, (const double*)D, Rv);
    else if (dtype == BLS_F32) jt_columns<float, 0>(P, g, (const float*)D, Rv);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_jtj_diag(bls_qr_plan* P, int dtype, double* d, const void* D) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (dtype == BLS_F64) jt_columns<double, 1>(P, d, (const double*)D, nullptr);
    else if (dtype == BLS_F32) jt_columns<float, 1>(P, d, (const float*)D, nullptr);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_jtj_quadform(bls_qr_plan* P, int dtype, const void* D, const double* v, double* result) {
  QR_GUARD({
    if (!P || !result) throw Error(BLS_EINVAL, "null argument");
    if (dtype == BLS_F64) *result = jtj_quadform<double>(P, (const double*)D, v);
    else if (dtype == BLS_F32) *result = jtj_quadform<float>(P, (const float*)D, v);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_assemble_hessian(bls_qr_plan* P, int dtype, const void* J, const double* r, void* E, void* C, void* R, int dense, double* b) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (dtype == BLS_F64) assemble<double>(P, (const double*)J, r, (double*)E, (double*)C, (double*)R, dense != 0, b);
    else if (dtype == BLS_F32) assemble<float>(P, (const float*)J, r, (float*)E, (float*)C, (float*)R, dense != 0, b);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_reduced_diagonal_blocks(bls_qr_plan* P, int dtype, void* D, const void* F) {
  QR_GUARD({
    if (dtype == BLS_F64) diagonal_blocks<double>(P, (double*)D, (const double*)F);
    else if (dtype == BLS_F32) diagonal_blocks<float>(P, (float*)D, (const float*)F);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}


int bls_reduced_residual(bls_qr_plan* P, const double* Fr, double* rt, int64_t n_rt) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (n_rt != P->red_nrows)
      throw Error(BLS_EDIM, "rt has length " + std::to_string(n_rt) + ", expected " + std::to_string(P->red_nrows));
    if (n_rt > 0 && (!Fr || !rt)) throw Error(BLS_EINVAL, "a device pointer is NULL");
    k_reduced_residual<<<(unsigned)std::max(1, grid_for(P->ntables * 32, 256)), 256, 0, P->ctx->stream>>>(
        P->ntables, P->t_rows.as<int32_t>(), P->t_top.as<int32_t>(), P->t_res.as<int64_t>(), P->t_red.as<int64_t>(), Fr, rt);
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

int bls_reduced_jacobian_dense(bls_qr_plan* P, int dtype, const void* F, const double* Fr, void* Jt, int64_t nrows, int64_t ncols,
                               double* rt, int64_t n_rt) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (nrows != P->red_nrows || ncols != P->nr)
      throw Error(BLS_EDIM, "Jt has size (" + std::to_string(nrows) + ", " + std::to_string(ncols) + "), expected (" +
                                std::to_string(P->red_nrows) + ", " + std::to_string(P->nr) + ")");
    if (n_rt != P->red_nrows)
      throw Error(BLS_EDIM, "rt has length " + std::to_string(n_rt) + ", expected " + std::to_string(P->red_nrows));
    if (P->red_nrows > 0 && (!F || !Fr || !Jt || !rt)) throw Error(BLS_EINVAL, "a device pointer is NULL");
    if (dtype == BLS_F64) reduced_jacobian_dense<double>(P, (double*)Jt, (const double*)F, Fr, rt);
    else if (dtype == BLS_F32) reduced_jacobian_dense<float>(P, (float*)Jt, (const float*)F, Fr, rt);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_reduced_jacobian_sparse(bls_qr_plan* P, int dtype, const void* F, const double* Fr, int64_t nrows, int64_t ncols,
                                const int64_t* colptr, const int64_t* rowval, void* nzval, double* rt, int64_t n_rt) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    check_jt_pattern(P, nrows, ncols, colptr, rowval);
    if (n_rt != P->red_nrows)
      throw Error(BLS_EDIM, "rt has length " + std::to_string(n_rt) + ", expected " + std::to_string(P->red_nrows));
    if (P->red_nrows > 0 && (!F || !Fr || !rt || (P->h_jt_colptr[P->nr] > 0 && !nzval))) throw Error(BLS_EINVAL, "a device pointer is NULL");
    if (dtype == BLS_F64) reduced_jacobian_sparse<double>(P, (double*)nzval, (const double*)F, Fr, rt);
    else if (dtype == BLS_F32) reduced_jacobian_sparse<float>(P, (float*)nzval, (const float*)F, Fr, rt);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}


int bls_reduced_mul(bls_qr_plan* P, int dtype, const void* F, const double* v, int64_t nv, double* y, int64_t ny) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (ny != P->red_nrows) throw Error(BLS_EDIM, "y has length " + std::to_string(ny) + ", expected " + std::to_string(P->red_nrows));
    if (nv != P->nr) throw Error(BLS_EDIM, "v has length " + std::to_string(nv) + ", expected " + std::to_string(P->nr));
    if (ny > 0 && (!F || !v || !y)) throw Error(BLS_EINVAL, "a device pointer is NULL");
    if (dtype == BLS_F64) launch_reduced_mul<double>(P, (const double*)F, v, y);
    else if (dtype == BLS_F32) launch_reduced_mul<float>(P, (const float*)F, v, y);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_reduced_tmul(bls_qr_plan* P, int dtype, const void* F, const double* w, int64_t nw, double* g, int64_t ng) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (ng != P->nr) throw Error(BLS_EDIM, "g has length " + std::to_string(ng) + ", expected " + std::to_string(P->nr));
    if (nw != P->red_nrows) throw Error(BLS_EDIM, "w has length " + std::to_string(nw) + ", expected " + std::to_string(P->red_nrows));
    if (ng > 0 && (!F || !w || !g)) throw Error(BLS_EINVAL, "a device pointer is NULL");
    if (dtype == BLS_F64) launch_reduced_tmul<double>(P, (const double*)F, w, g);
    else if (dtype == BLS_F32) launch_reduced_tmul<float>(P, (const float*)F, w, g);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_lsmr_reduced(bls_qr_plan* P, int dtype, const void* F, const double* Fr, double lambda, const double* s_r, double* x,
                     int64_t nx, double atol, double btol, double conlim, int64_t itmax, int64_t* iterations, int* istop,
                     double* stats) {
  QR_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (nx != P->nr) throw Error(BLS_EDIM, "x has length " + std::to_string(nx) + ", expected " + std::to_string(P->nr));
    if (P->nr > 0 && (!F || !x || (P->red_nrows > 0 && !Fr))) throw Error(BLS_EINVAL, "a device pointer is NULL");
    if (!(lambda >= 0) || !(atol >= 0) || !(btol >= 0) || !(conlim >= 0))
      throw Error(BLS_EINVAL, "lambda, atol, btol and conlim must be non-negative");
    if (itmax < 0) itmax = P->red_nrows + P->nr;
    LsmrOut o;
    int rc;
    if (dtype == BLS_F64) rc = lsmr_reduced<double>(P, (const double*)F, Fr, lambda, s_r, x, atol, btol, conlim, itmax, &o);
    else if (dtype == BLS_F32) rc = lsmr_reduced<float>(P, (const float*)F, Fr, lambda, s_r, x, atol, btol, conlim, itmax, &o);
    else throw Error(BLS_EINVAL, "unknown dtype");
    if (iterations) *iterations = o.iterations;
    if (istop) *istop = o.istop;
    if (stats) {
      stats[0] = o.normr;
      stats[1] = o.normar;
      stats[2] = o.normA;
      stats[3] = o.condA;
      stats[4] = o.normx;
    }
    return rc;
  })
}

}  // extern "C"
