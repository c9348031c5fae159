// Schur-complement elimination of the point blocks on sm_100a.
//
// Reference: src/schur_reduction.jl (SchurReductionWorkspace :16-92, factor_eliminated! :121-162, accumulate_entry_*!
// :262-354, reset_schur_*! :389-436, reduce_schur_*! :465-507, backsubstitute! :519-576), src/kernels.jl:3-67
// (inv_sym_block), src/conditioning.jl:99-150 (scaling at read).
//
// Device layout. Everything the reference keeps in its workspace is built once per structure into a plan:
//   - the structure's index arrays as int32 (r_dims, boffsets, eliminated_ptr, entry_retained, coffsets, ...);
//   - the S blocks that receive contributions, each with the base index of its (0, 0) entry and its column stride
//     (sparse: S_colptr[boffsets_r[r2]] + block_row_offsets[k] and col_heights[r2]; dense: the column-major offset
//     and nr), so one kernel serves reduce_schur_sparse! and reduce_schur_dense!;
//   - for every S block (r1, r2) the list of coupling pairs (c1, c2) of the points that observe both (c1 of r1, c2 of
//     r2, same point), in ascending point order, cut into work items of at most PAIR_CHUNK pairs.
// A call then runs:
//   phase 1  k_factor   one thread per point: the damped d_e x d_e inverse in FP64 (closed forms of
//                        src/kernels.jl:14-67, same pivot tests), z = E^-1 (s_e .* b_e) in FP64;
//   phase 2  k_pairs    one thread per work item: sum over its pairs of C_c1' (E^-1 C_c2), the 6x6 block in
//                        registers, then one plain read-modify-write of S when the block has a single item, else
//                        atomic adds (one per block entry per item, not per pair);
//            k_gradient one warp per retained block: g_S = s_r .* b_r - sum C' z over its couplings.
// The reference forms W = E^-1 C in phase 1 and reads it back in phase 2; here E^-1 C_c2 is formed in registers
// where it is used, so nothing the size of C_data is written. W' C and C' (E^-1 C) are the same product (E^-1 is
// symmetric); the order of the additions differs, which the tests bound by tolerance.
#include <algorithm>
#include <cstdio>
#include <climits>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <omp.h>
#include <type_traits>

#include "closed_inverse.cuh"
#include "common.cuh"

namespace bls {

constexpr int PAIR_CHUNK = 32;
constexpr long long NONE = LLONG_MAX;

// ------------------------------------------------------------------------------------------------------------------
// Plan
// ------------------------------------------------------------------------------------------------------------------
struct SchurPlan {
  bls_ctx* ctx = nullptr;
  int64_t nrblocks = 0, neblocks = 0, nr = 0, ne = 0, ncoup = 0, E_length = 0, C_length = 0;
  int64_t nblocks = 0, npairs = 0, nitems = 0, nnzS = 0, R_length = 0;
  bool has_sparse = false;
  int max_de = 0, max_dr = 0;
  bool uniform36 = false;   // every r_dim is 6 and every e_dim is 3
  bool fast36 = false;      // uniform36 with the canonical offsets (coffsets = 18c, eoffsets = 9e) and packable pairs
  std::vector<int64_t> diag_inds_host;
  // structure
  DevBuf r_dims, boffsets_r, e_dims, boffsets_e, eoffsets, eliminated_ptr, entry_retained, coffsets, entry_eliminated;
  DevBuf retained_ptr, retained_entry;
  // blocks and pairs
  DevBuf block_r1, block_r2, block_base_sparse, block_stride_sparse, block_base_dense;
  DevBuf pair_c1, pair_c2, item_block, item_start, item_info;
  DevBuf pair_packed;   // fast36: {c1, e | (c2 - c1) << 24} per pair
  // fast36, column kernel: per visit {p0, e | j << 24} and the start of its row offsets; per (visit, camera) the
  // camera's row offset in the column's tile; per column the S index of its first entry
  DevBuf vis_rec, vis_base, vis_off, col_base, col_h;
  int64_t max_col_h = 0;
  bool tiles_ok = false;   // every point's coupling span fits the staging buffer of k_tiles36
  DevBuf pt_rec;   // fast36, point-major pairs: {c1, k | (c2 - c1) << 25} per pair, k the S block
  bool points_ok = false;
  // fast36, sparse: the column-owned schedule (k_stage36). Work items are runs of a block column's visits (most
  // columns are one item); per item {r2, first visit, visit count, items of its column} (stg_items) and its first
  // batch (stg_ibat, nitems + 1). The diagonal block is formed by the staging pass (no batch);
  // the item's off-diagonal pairs are cut into units (one S block, at most stage_unit[sd] pairs, in visit order), and those units,
  // longest first, into the following batches of 32, one unit per lane of the warp that takes the batch: per batch
  // {first pair, iterations} (stg_bat), per batch and lane {the block's row offset in the column | unit length << 16 |
  // (the block's only unit in the item) << 31} (stg_lane); pairs batch by batch, iteration-major (lane fastest),
  // {visit within the item | c1's index within its point << 16}, 0 past a lane's unit (stg_pairs).
  // One schedule per storage type (index 0 FP32, 1 FP64): FP32 items fit two 256-thread CTAs per SM, FP64 items (half
  // the visits) two 128-thread CTAs.
  bool stage_ok = false;
  // per schedule, the unit size (measured on the 1M-point scene: FP32 1.73 ms at 16, 1.62 at 20, 1.68 at 24; FP64
  // 3.07 ms at 16, 3.30 at 20; on the 200k-point scene FP32 0.318 / 0.303 / 0.300 ms and FP64 0.468 ms at 16)
  int stage_unit[2] = {20, 16};
  struct StageSchedule {
    int64_t items = 0, max_nv = 0, units = 0, batches = 0, slots = 0;
    DevBuf stg_items, stg_ibat, stg_bat, stg_lane, stg_pairs;
  };
  StageSchedule stage[2];
  int stage_grid[2] = {0, 0};   // persistent CTAs of k_stage36 (FP32, FP64): resident blocks per SM x SMs
  DevBuf EZ;   // per point E' = s_e E^-1 s_e (9, column-major) and z' = s_e .* z (3), FP64, for k_stage36
  // a batch of independent problems in one plan (bls_schur_plan_set_problems): per problem the lowest failing point
  // (global index, NONE if none), per point and per camera its problem; a failing problem skips its own phase 2 only
  int64_t nprob = 0;
  std::vector<int64_t> prob_point_off, prob_row_off, prob_nnz_off;
  DevBuf prob_fail, prob_of_point, prob_of_cam;
  int kernel = 1;   // 0: column-owned (k_columns36), 1: block-owned pairs (k_pairs36, the default: faster on sparse scenes)
  // reset
  DevBuf r_to_s, diag_inds, S_rowval, S_col;
  // one-pass reset (k_reset_columns): per S entry the R entry it takes or -1, and S's column pointers; used when
  // every diag_inds[i] lies in column i
  DevBuf r_from, S_colptr;
  bool reset_fused = false;
  // host-buffer reduction (fast36, sparse): the points cut into stages of about equal coupling count, and the pair
  // work items re-cut so that each item's pairs lie in one stage (stage j: items [stage_item[j], stage_item[j + 1]))
  static constexpr int kStages = 16;
  bool staged = false;
  int64_t stage_pt[kStages + 1] = {}, stage_cp[kStages + 1] = {}, stage_item[kStages + 1] = {};
  DevBuf st_block, st_start, st_info;
  // device copies of the host call's inputs and outputs (allocated at its first call), its copy stream and events
  DevBuf h_E, h_C, h_R, h_br, h_be, h_scr, h_sce, h_S, h_g;
  size_t h_elem = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_free = nullptr, ev_points = nullptr, ev_in[kStages + 1] = {};
  // scratch: E^-1 (FP64, and FP32 for the mixed form), z, status
  DevBuf Einv64, Einv32, z, status;
  DevBuf acc1;     // one FP64 accumulator (bls_hessian_bilinear)
  DevBuf w_apply;  // per point E^-1 C x of bls_schur_apply_elimination (ne doubles, allocated at its first call)
  DevBuf t_apply;  // per point C x of bls_schur_apply_elimination on the 3-variable fast path (3 neblocks doubles)
  DevBuf Einv12;   // fast36: E^-1 per point in the element type of the pair products, padded to 12 entries (16-byte rows)
  Status* host_status = nullptr;   // pinned
  int last_dtype = -1;
  // instrumentation: launches issued on the plan, and CUDA events around the pair kernel when timing is on
  int64_t launches = 0;
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pair_events;
  ~SchurPlan() {
    if (host_status) cudaFreeHost(host_status);
    if (ev_free) cudaEventDestroy(ev_free);
    if (ev_points) cudaEventDestroy(ev_points);
    for (auto& e : ev_in) if (e) cudaEventDestroy(e);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (auto& e : pair_events) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  }
};

static std::vector<int32_t> to32(const int64_t* a, int64_t n, const char* what) {
  std::vector<int32_t> v((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    if (a[i] < INT32_MIN || a[i] > INT32_MAX) throw Error(BLS_EUNSUPPORTED, std::string(what) + " exceeds the 32-bit index range of this build");
    v[i] = (int32_t)a[i];
  }
  return v;
}

// ------------------------------------------------------------------------------------------------------------------
// Kernels
// ------------------------------------------------------------------------------------------------------------------
// which = 0: the reset's scaling_r slot; 1: the reduction's scaling_e slot
__global__ void k_status_begin(Status* st, int which) {
  if (which == 0) st->einval_r = NONE;
  else st->einval_e = NONE;
}
// check_damping (src/utils.jl:100-107): every scaling entry finite and non-negative; the lowest bad index is kept
__global__ void k_check_scaling(const double* __restrict__ sc, int64_t n, Status* st, int which) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = sc[i];
  if (!(isfinite(x) && x >= 0.0)) atomicMin(which == 0 ? &st->einval_r : &st->einval_e, (long long)i);
}
__device__ __forceinline__ bool args_ok(const Status* st) { return st->einval_r == NONE && st->einval_e == NONE; }
// The reduction's failure word starts clear when the arguments are valid
__global__ void k_arm(Status* st) {
  if (args_ok(st)) st->failed = NONE;
}

__device__ __forceinline__ bool live(const Status* st) { return args_ok(st) && st->failed == NONE; }

// --- reset_schur_sparse!: fill, scatter R by the r -> s map, scale, damp the diagonal ---
template <class T>
__global__ void k_fill(T* __restrict__ S, int64_t n, const Status* st) {
  if (st->einval_r != NONE) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) S[i] = T(0);
}
template <class T>
__global__ void k_scatter_r(T* __restrict__ S, const T* __restrict__ R, const int64_t* __restrict__ map, int64_t n, const Status* st) {
  if (st->einval_r != NONE) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t idx = map[i];
    if (idx >= 0) S[idx] = R[i];
  }
}
// scale_sparse! (src/conditioning.jl:144-150): nz = T(nz * s[row] * s[col]), formed in FP64
template <class T>
__global__ void k_scale_sparse(T* __restrict__ S, const int32_t* __restrict__ rowval, const int32_t* __restrict__ col,
                               const double* __restrict__ s, int64_t n, const Status* st) {
  if (st->einval_r != NONE) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) S[i] = T((double)S[i] * (s[rowval[i]] * s[col[i]]));
}
// nzval[idx] = T(Float64(nzval[idx]) + lambda * scaling_r[i] * (s_i * s_i)) (src/schur_reduction.jl:430-433)
template <class T>
__global__ void k_damp_diag(T* __restrict__ S, const int64_t* __restrict__ diag_inds, int64_t dense_nr,
                            const double* __restrict__ sc, double lambda, const double* __restrict__ s, int64_t nr, Status* st) {
  if (st->einval_r != NONE) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nr) return;
  double si = s ? s[i] : 1.0;
  int64_t idx = diag_inds ? diag_inds[i] : i * (dense_nr + 1);
  S[idx] = T((double)S[idx] + lambda * sc[i] * (si * si));
}
// reset_schur_dense! copy with scaling (src/schur_reduction.jl:394-400)
template <class T>
__global__ void k_copy_scaled_dense(T* __restrict__ S, const T* __restrict__ R, const double* __restrict__ s, int64_t nr, const Status* st) {
  if (st->einval_r != NONE) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < nr * nr; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = i % nr, c = i / nr;
    S[i] = s ? T((double)R[i] * (s[r] * s[c])) : R[i];
  }
}
__global__ void k_reset_done(Status* st) {
  if (st->einval_r == NONE) st->failed = NONE;
}

// check_damping for short vectors in one block, without a separate clearing launch: the lowest index whose entry is
// negative or not finite (NONE if none) is written to the slot (which = 0: scaling_r, 1: scaling_e).
__global__ void __launch_bounds__(1024) k_check_scaling1(const double* __restrict__ sc, int64_t n, Status* st, int which) {
  __shared__ long long lowest;
  if (threadIdx.x == 0) lowest = NONE;
  __syncthreads();
  long long m = NONE;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = sc[i];
    if (!(isfinite(x) && x >= 0.0) && i < m) m = i;
  }
  if (m != NONE) atomicMin(&lowest, m);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (which == 0) st->einval_r = lowest;
    else st->einval_e = lowest;
  }
}

// reset_schur_sparse! (src/schur_reduction.jl:416-436) in one pass: one warp per column j of S. Entry q takes
// R[r_from[q]] (zero when no R entry maps there; r_from keeps the last entry of the map that does, as the reference's
// loop leaves it), scaled by T(v * (s_r[row] * s_r[j])) when conditioned; then lane 0 damps the column's diagonal
// entry diag_inds[j] (inside the column, so no other warp touches it). Warp 0 also clears the failure word, as the
// reference's ws.failed_block[] = 0. scaling_r was checked by the kernel before.
template <class T>
__global__ void __launch_bounds__(256) k_reset_columns(T* __restrict__ S, const T* __restrict__ R, const int32_t* __restrict__ r_from,
                                                     const int64_t* __restrict__ colptr, const int32_t* __restrict__ rowval,
                                                     const int64_t* __restrict__ diag_inds, const double* __restrict__ sc, double lambda,
                                                     const double* __restrict__ s_r, int64_t nr, Status* st) {
  const int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (st->einval_r != NONE) return;
  if (j == 0 && lane == 0) st->failed = NONE;
  if (j >= nr) return;
  const int64_t q0 = colptr[j], q1 = colptr[j + 1];
  const double sj = s_r ? s_r[j] : 1.0;
  for (int64_t q = q0 + lane; q < q1; q += 32) {
    const int32_t i = r_from[q];
    T v = i >= 0 ? R[i] : T(0);
    if (s_r) v = T((double)v * (s_r[rowval[q]] * sj));
    S[q] = v;
  }
  __syncwarp();
  if (lane == 0) {
    const int64_t d = diag_inds[j];
    S[d] = T((double)S[d] + lambda * sc[j] * (sj * sj));
  }
}

// reset_schur_dense! (src/schur_reduction.jl:389-407) in one pass: one warp per column j, S[:, j] = R[:, j] (scaled
// by T(R * (s_r[i] * s_r[j])) when conditioned), then lane 0 damps S[j, j]; warp 0 clears the failure word.
template <class T>
__global__ void __launch_bounds__(256) k_reset_dense_columns(T* __restrict__ S, const T* __restrict__ R, const double* __restrict__ sc,
                                                           double lambda, const double* __restrict__ s_r, int64_t nr, Status* st) {
  const int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (st->einval_r != NONE) return;
  if (j == 0 && lane == 0) st->failed = NONE;
  if (j >= nr) return;
  const double sj = s_r ? s_r[j] : 1.0;
  for (int64_t i = lane; i < nr; i += 32) S[i + nr * j] = s_r ? T((double)R[i + nr * j] * (s_r[i] * sj)) : R[i + nr * j];
  __syncwarp();
  if (lane == 0) S[j + nr * j] = T((double)S[j + nr * j] + lambda * sc[j] * (sj * sj));
}

// The reduction's status for the 6/3 fast path: scaling_e is checked by k_factor36 itself, so its slot is cleared
// here, and the failure word is cleared when the reset's arguments were valid.
__global__ void k_arm36(Status* st) {
  st->einval_e = NONE;
  if (st->einval_r == NONE) st->failed = NONE;
  st->pad = 0;   // the work queue of k_stage36
}

template <class T>
__global__ void __launch_bounds__(256) k_factor(int64_t neb, const int32_t* __restrict__ e_dims, const int32_t* __restrict__ eoffsets,
                                                const int32_t* __restrict__ boffsets_e, const T* __restrict__ E,
                                                const double* __restrict__ b_e, const double* __restrict__ scaling_e, double lambda,
                                                const double* __restrict__ s_e, double* __restrict__ Einv64, float* __restrict__ Einv32,
                                                double* __restrict__ z, Status* st) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb) return;
  if (!args_ok(st)) return;
  const int de = e_dims[e], eo = eoffsets[e], so = boffsets_e[e];
  double se[16], damp[16], H[256], inv[256];
  for (int i = 0; i < de; ++i) {
    se[i] = s_e ? s_e[so + i] : 1.0;
    damp[i] = mul(mul(lambda, scaling_e[so + i]), mul(se[i], se[i]));
  }
  for (int j = 0; j < de; ++j)
    for (int i = 0; i < de; ++i) {
      double h = (double)E[eo + i + de * j];
      H[i + de * j] = s_e ? mul(h, mul(se[i], se[j])) : h;
    }
  if (!(de <= 3 ? inv_sym_closed(de, H, damp, inv) : inv_sym_chol(de, H, damp, inv))) {
    atomicMin(&st->failed, (long long)e);
    return;
  }
  for (int i = 0; i < de * de; ++i) {
    Einv64[eo + i] = inv[i];
    if (Einv32) Einv32[eo + i] = (float)inv[i];
  }
  for (int i = 0; i < de; ++i) {
    double acc = inv[i] * (b_e[so] * se[0]);
    for (int j = 1; j < de; ++j) acc = acc + inv[i + de * j] * (b_e[so + j] * se[j]);
    z[so + i] = acc;
  }
}

// element type of the E^-1 copy the pair products read: FP32 in the mixed form, FP64 otherwise
template <class T> struct EinvOf { using type = double; };
template <> struct EinvOf<float> { using type = float; };

// factor_eliminated! for the fast path (d_e = 3, canonical layout: point e's E block at 9 e, its variables at 3 e):
// the same per-point arithmetic as k_factor, with a block's 128 points staged through shared memory so that E, b_e,
// scaling_e and s_e are read, and E^-1 (FP64), the padded E^-1 of the pair products and z are written, in contiguous
// coalesced runs instead of one 36-72-byte run per thread. The FP32 copy of E^-1 that only the generic phase 2 reads
// is not written. It also applies check_damping to scaling_e (the lowest bad entry into the status word), so the
// reduction needs no separate checking launch; the pair kernel that follows skips its work if any entry was bad.
template <class T>
__global__ void __launch_bounds__(128) k_factor36(int64_t e_begin, int64_t neb, const T* __restrict__ E, const double* __restrict__ b_e,
                                                  const double* __restrict__ scaling_e, double lambda, const double* __restrict__ s_e,
                                                  double* __restrict__ Einv64, typename EinvOf<T>::type* __restrict__ Einv12,
                                                  double* __restrict__ z, double* __restrict__ EZ, const int32_t* __restrict__ prob_of_point,
                                                  long long* __restrict__ prob_fail, Status* st) {
  using TE = typename EinvOf<T>::type;
  constexpr int NB = 128;
  __shared__ double sE[NB * 9];      // E in, then E^-1 out
  __shared__ TE s12[NB * 12];
  __shared__ double sb[NB * 3], ss[NB * 3], sse[NB * 3];
  __shared__ double sez[NB * 12];    // k_stage36's record: E' = s_e E^-1 s_e and z' = s_e .* z
  if (st->einval_r != NONE) return;   // the reset's arguments were bad; scaling_e is checked here (k_arm36 cleared its slot)
  const int64_t e0 = e_begin + (int64_t)blockIdx.x * NB;   // points [e_begin, neb)
  const int n = (int)(neb - e0 < NB ? neb - e0 : NB);
  const int t = threadIdx.x;
  for (int i = t; i < 9 * n; i += NB) sE[i] = (double)E[9 * e0 + i];
  for (int i = t; i < 3 * n; i += NB) {
    sb[i] = b_e[3 * e0 + i];
    const double x = scaling_e[3 * e0 + i];
    if (!(isfinite(x) && x >= 0.0)) atomicMin(&st->einval_e, (long long)(3 * e0 + i));   // check_damping, src/utils.jl:100-107
    ss[i] = x;
    sse[i] = s_e ? s_e[3 * e0 + i] : 1.0;
  }
  __syncthreads();
  if (t < n) {
    double se[3], damp[3], H[9], inv[9];
    for (int i = 0; i < 3; ++i) {
      se[i] = sse[3 * t + i];
      damp[i] = mul(mul(lambda, ss[3 * t + i]), mul(se[i], se[i]));
    }
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        const double h = sE[9 * t + i + 3 * j];
        H[i + 3 * j] = s_e ? mul(h, mul(se[i], se[j])) : h;
      }
    if (!inv_sym_closed(3, H, damp, inv)) {
      if (prob_fail) atomicMin(prob_fail + prob_of_point[e0 + t], (long long)(e0 + t));   // this problem's lowest failing point
      else atomicMin(&st->failed, (long long)(e0 + t));
      for (int i = 0; i < 9; ++i) inv[i] = 0.0;
    }
    for (int i = 0; i < 9; ++i) {
      sE[9 * t + i] = inv[i];
      s12[12 * t + i] = (TE)inv[i];
    }
    for (int i = 9; i < 12; ++i) s12[12 * t + i] = TE(0);
    for (int i = 0; i < 3; ++i) {
      double acc = inv[i] * (sb[3 * t] * se[0]);
      for (int j = 1; j < 3; ++j) acc = acc + inv[i + 3 * j] * (sb[3 * t + j] * se[j]);
      ss[3 * t + i] = acc;     // z, in the slot of scaling_e (read above by this thread only)
      sez[12 * t + 9 + i] = se[i] * acc;
    }
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) sez[12 * t + i + 3 * j] = se[i] * inv[i + 3 * j] * se[j];
  }
  __syncthreads();
  for (int i = t; i < 9 * n; i += NB) Einv64[9 * e0 + i] = sE[i];
  if (Einv12)
    for (int i = t; i < 12 * n; i += NB) Einv12[12 * e0 + i] = s12[i];
  if (EZ)
    for (int i = t; i < 12 * n; i += NB) EZ[12 * e0 + i] = sez[i];
  for (int i = t; i < 3 * n; i += NB) z[3 * e0 + i] = ss[i];
}

// dot(x, H, y) / schur_bilinear (src/linalg.jl:133-262) from a SchurBlockHessian with R on S's pattern: x'Hy, FP64,
// each stored off-diagonal entry counted in both orientations (a_x b_y + a_y b_x), as the reference's walk of one
// stored triangle does. Retained part: one thread per stored entry (upper part; the lower entries of the diagonal
// blocks are not part of R); point part: one thread per eliminated block (its E block and coupling blocks). Partial
// sums per warp, one FP64 atomic per warp.
__device__ __forceinline__ double warp_sum_h(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <class T>
__global__ void k_bilinear_R(int64_t nnz, int64_t dense_nr, const int32_t* __restrict__ rowval, const int32_t* __restrict__ colof,
                             const T* __restrict__ R, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ out) {
  double part = 0.0;
  const int64_t n = dense_nr ? dense_nr * dense_nr : nnz;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = dense_nr ? q % dense_nr : rowval[q], j = dense_nr ? q / dense_nr : colof[q];
    if (i > j) continue;
    const double v = (double)R[q];
    part += i == j ? v * x[i] * y[i] : v * (x[i] * y[j] + x[j] * y[i]);
  }
  part = warp_sum_h(part);
  if ((threadIdx.x & 31) == 0 && part != 0.0) atomicAdd(out, part);
}
template <class T>
__global__ void k_bilinear_points(int64_t neb, int64_t nr, const int32_t* __restrict__ eliminated_ptr, const int32_t* __restrict__ entry_retained,
                                  const int32_t* __restrict__ e_dims, const int32_t* __restrict__ eoffsets, const int32_t* __restrict__ boffsets_e,
                                  const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boffsets_r, const int32_t* __restrict__ coffsets,
                                  const T* __restrict__ E, const T* __restrict__ C, const double* __restrict__ x, const double* __restrict__ y,
                                  double* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double part = 0.0;
  if (e < neb) {
    const int de = e_dims[e], eo = eoffsets[e];
    const double* xe = x + nr + boffsets_e[e];
    const double* ye = y + nr + boffsets_e[e];
    for (int b = 0; b < de; ++b)
      for (int a = 0; a < de; ++a) part += xe[a] * (double)E[eo + a + de * b] * ye[b];
    for (int c = eliminated_ptr[e]; c < eliminated_ptr[e + 1]; ++c) {
      const int r = entry_retained[c], dr = r_dims[r], ro = boffsets_r[r], co = coffsets[c];
      for (int w = 0; w < dr; ++w)
        for (int a = 0; a < de; ++a) {
          const double h = (double)C[co + a + de * w];
          part += h * (xe[a] * y[ro + w] + ye[a] * x[ro + w]);
        }
    }
  }
  part = warp_sum_h(part);
  if ((threadIdx.x & 31) == 0 && part != 0.0) atomicAdd(out, part);
}
// The diagonal of H (the `diag!` a conditioned Hessian system hands prepare_scale!): d = [diag R; diag of each E block]
template <class T>
__global__ void k_hessian_diag(int64_t nr, int64_t neb, const int64_t* __restrict__ diag_inds, int64_t dense_nr, const int32_t* __restrict__ e_dims,
                               const int32_t* __restrict__ eoffsets, const int32_t* __restrict__ boffsets_e, const T* __restrict__ R,
                               const T* __restrict__ E, double* __restrict__ d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < nr) d[i] = (double)R[dense_nr ? i + dense_nr * i : diag_inds[i]];
  if (i < neb) {
    const int de = e_dims[i];
    for (int a = 0; a < de; ++a) d[nr + boffsets_e[i] + a] = (double)E[eoffsets[i] + a + de * a];
  }
}

// --- phase 2: one thread per work item of one S block ---

template <class T>
__device__ __forceinline__ void red_add(T* p, T v) { atomicAdd(p, v); }

// MDE/MDR: compile-time bounds of d_e and d_r; the runtime sizes are checked against them by the host.
template <class T, int MDE, int MDR>
__global__ void __launch_bounds__(128) k_pairs(
    int64_t nitems, const int32_t* __restrict__ item_block, const int32_t* __restrict__ item_start, const int32_t* __restrict__ item_info,
    const int32_t* __restrict__ pair_c1, const int32_t* __restrict__ pair_c2, const int32_t* __restrict__ block_r1,
    const int32_t* __restrict__ block_r2, const int64_t* __restrict__ block_base, const int32_t* __restrict__ block_stride, int64_t dense_nr,
    const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boffsets_r, const int32_t* __restrict__ entry_eliminated,
    const int32_t* __restrict__ e_dims, const int32_t* __restrict__ boffsets_e, const int32_t* __restrict__ eoffsets,
    const int32_t* __restrict__ coffsets, const T* __restrict__ C, const typename EinvOf<T>::type* __restrict__ Einv,
    const double* __restrict__ s_r, const double* __restrict__ s_e, T* __restrict__ S, const Status* __restrict__ st) {
  using TE = typename EinvOf<T>::type;
  const int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (it >= nitems) return;
  if (!live(st)) return;
  const int k = item_block[it], p_begin = item_start[it], info = item_info[it];
  const int cnt = info & 0xffff;
  const bool solo = (info >> 16) != 0;
  const int r1 = block_r1[k], r2 = block_r2[k];
  const bool diag = r1 == r2;
  const int d1 = r_dims[r1], d2 = r_dims[r2], ro1 = boffsets_r[r1], ro2 = boffsets_r[r2];
  T acc[MDR][MDR];
#pragma unroll
  for (int a = 0; a < MDR; ++a)
#pragma unroll
    for (int b = 0; b < MDR; ++b) acc[a][b] = T(0);
  for (int p = p_begin; p < p_begin + cnt; ++p) {
    const int c1 = pair_c1[p], c2 = pair_c2[p];
    const int e = entry_eliminated[c2];
    const int de = e_dims[e], so = boffsets_e[e], eo = eoffsets[e];
    const int co1 = coffsets[c1], co2 = coffsets[c2];
    double se[MDE];
#pragma unroll
    for (int s = 0; s < MDE; ++s) se[s] = (s < de && s_e) ? s_e[so + s] : 1.0;
    TE Ei[MDE][MDE];
#pragma unroll
    for (int a = 0; a < MDE; ++a)
#pragma unroll
      for (int b = 0; b < MDE; ++b) Ei[a][b] = (a < de && b < de) ? Einv[eo + a + de * b] : TE(0);
    // U = E^-1 * scaled(C_c2)  (d_e x d2)
    T U[MDE][MDR];
#pragma unroll
    for (int w = 0; w < MDR; ++w) {
      T cw[MDE];
      const double fw = (w < d2 && s_r) ? s_r[ro2 + w] : 1.0;
#pragma unroll
      for (int s = 0; s < MDE; ++s) {
        T c = (w < d2 && s < de) ? C[co2 + w * de + s] : T(0);
        cw[s] = (s_r || s_e) ? T((double)c * (se[s] * fw)) : c;
      }
#pragma unroll
      for (int t = 0; t < MDE; ++t) {
        TE u = TE(0);
#pragma unroll
        for (int s = 0; s < MDE; ++s) u = u + Ei[t][s] * (TE)cw[s];
        U[t][w] = (T)u;
      }
    }
    // acc += scaled(C_c1)' * U
#pragma unroll
    for (int rho = 0; rho < MDR; ++rho) {
      T cr[MDE];
      const double fr = (rho < d1 && s_r) ? s_r[ro1 + rho] : 1.0;
#pragma unroll
      for (int s = 0; s < MDE; ++s) {
        T c = (rho < d1 && s < de) ? C[co1 + rho * de + s] : T(0);
        cr[s] = (s_r || s_e) ? T((double)c * (se[s] * fr)) : c;
      }
#pragma unroll
      for (int w = 0; w < MDR; ++w) {
        T a = acc[rho][w];
#pragma unroll
        for (int s = 0; s < MDE; ++s) a = a + cr[s] * U[s][w];
        acc[rho][w] = a;
      }
    }
  }
  const int64_t base = block_base[k];
  const int64_t stride = block_stride ? (int64_t)block_stride[k] : dense_nr;
#pragma unroll
  for (int w = 0; w < MDR; ++w) {
    if (w >= d2) continue;
#pragma unroll
    for (int rho = 0; rho < MDR; ++rho) {
      if (rho >= d1 || (diag && rho > w)) continue;
      T* p = S + base + w * stride + rho;
      if (solo) *p = *p - acc[rho][w];
      else red_add(p, -acc[rho][w]);
    }
  }
}

// g_S = s_r .* b_r - sum over the couplings c2 of r2 of scaled(C_c2)' z_e (src/schur_reduction.jl:326-328, 473/500)
template <class T>
__global__ void __launch_bounds__(256) k_gradient(int64_t nrb, const int32_t* __restrict__ retained_ptr, const int32_t* __restrict__ retained_entry,
                                                  const int32_t* __restrict__ entry_eliminated, const int32_t* __restrict__ r_dims,
                                                  const int32_t* __restrict__ boffsets_r, const int32_t* __restrict__ e_dims,
                                                  const int32_t* __restrict__ boffsets_e, const int32_t* __restrict__ coffsets,
                                                  const T* __restrict__ C, const double* __restrict__ z, const double* __restrict__ b_r,
                                                  const double* __restrict__ s_r, const double* __restrict__ s_e, double* __restrict__ g,
                                                  const Status* __restrict__ st) {
  const int64_t r2 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r2 >= nrb) return;
  if (!live(st)) return;
  const int d2 = r_dims[r2], ro2 = boffsets_r[r2];
  double acc[16];
  for (int w = 0; w < 16; ++w) acc[w] = 0.0;
  for (int q = retained_ptr[r2] + lane; q < retained_ptr[r2 + 1]; q += 32) {
    const int c2 = retained_entry[q], e = entry_eliminated[c2];
    const int de = e_dims[e], so = boffsets_e[e], co = coffsets[c2];
    for (int w = 0; w < d2 && w < 16; ++w) {
      const double f = s_r ? s_r[ro2 + w] : 1.0;
      double d = 0.0;
      for (int s = 0; s < de; ++s) {
        T c = C[co + w * de + s];
        double cs = (s_r || s_e) ? (double)T((double)c * ((s_e ? s_e[so + s] : 1.0) * f)) : (double)c;
        d = d + cs * z[so + s];
      }
      acc[w] += d;
    }
  }
  for (int w = 0; w < 16; ++w)
    for (int off = 16; off > 0; off >>= 1) acc[w] += __shfl_xor_sync(0xffffffffu, acc[w], off);
  if (lane < d2 && lane < 16) {
    double bv = b_r[ro2 + lane];
    if (s_r) bv = bv * s_r[ro2 + lane];
    double a = 0.0;
    for (int w = 0; w < 16; ++w) if (w == lane) a = acc[w];
    g[ro2 + lane] = bv - a;
  }
}

// g_S = s_r .* b_r (scaled_copy!, src/conditioning.jl:237-244), before the pair kernel subtracts C' z
__global__ void k_g_init(double* __restrict__ g, const double* __restrict__ b_r, const double* __restrict__ s_r, int64_t nr,
                         const Status* __restrict__ st, const int32_t* __restrict__ prob_of_cam = nullptr,
                         const long long* __restrict__ prob_fail = nullptr) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nr || !live(st)) return;
  if (prob_fail && prob_fail[prob_of_cam[i / 6]] != NONE) return;   // a failing problem keeps its g_S
  g[i] = s_r ? b_r[i] * s_r[i] : b_r[i];
}
__global__ void k_prob_arm(long long* __restrict__ prob_fail, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) prob_fail[i] = NONE;
}

// Column w of a 3 x 6 coupling block in the canonical layout: three entries starting at 18 c + 3 w, which is even
// exactly when w is (odd = w & 1). FP64: one 16-byte load at the even offset and one single load cover them, with
// no divergence between the parities (C is aligned to two elements); 0.557 -> 0.539 ms on the 200k-point scene.
// FP32: three single loads (the paired form measured slower there, 0.341 -> 0.368 ms).
__device__ __forceinline__ void load_col3(const float* p, int, float out[3]) {
  out[0] = __ldg(p);
  out[1] = __ldg(p + 1);
  out[2] = __ldg(p + 2);
}
__device__ __forceinline__ void load_col3(const double* p, int odd, double out[3]) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p + odd));
  const double s = __ldg(p + (odd ? 0 : 2));
  out[0] = odd ? s : v.x;
  out[1] = odd ? v.x : v.y;
  out[2] = odd ? v.y : s;
}

// Phase 2 for d_r = 6, d_e = 3 in the canonical layout (coffsets = 18 c, eoffsets = 9 e): six threads per work item,
// thread w accumulating column w of the 6 x 6 block, so the block's state is 6 values per thread rather than 36. Per
// pair a thread loads the point's E^-1 (padded row of 12), all of C_c1 and column w of C_c2, forms u = E^-1 C_c2[:, w]
// and adds C_c1' u to its column. A pair record {c1, e | (c2 - c1) << 24} holds every index the pair needs, so the
// next record is fetched while the current pair is computed and no load waits on another index load. The diagonal
// block's items also subtract C_c2' z from g_S (each coupling of r2 is exactly one diagonal pair).
// The same two passes for the 6/3 canonical layout (C_c at 18 c, E^-1 at 9 e, variables at 6 r and 3 e): no per-block
// index loads, each coupling block read with 8- or 16-byte loads and each x_r block with 16-byte loads, two couplings
// of a point in flight at a time. Pass 1, one thread per point: w_e = E^-1 sum_c C_c x_r(c). Pass 2, one warp per
// camera, lanes over its couplings: y_r = y0_r - sum_c C_c' w_e(c), six sums reduced across the warp.
template <class T>
__device__ __forceinline__ void coupling18(const T* __restrict__ C, int64_t c, T out[18]) {
  if constexpr (std::is_same<T, double>::value) {
    const double2* q = reinterpret_cast<const double2*>(C + 18 * c);
#pragma unroll
    for (int i = 0; i < 9; ++i) { const double2 v = __ldg(q + i); out[2 * i] = v.x; out[2 * i + 1] = v.y; }
  } else {
    const float2* q = reinterpret_cast<const float2*>(C + 18 * c);
#pragma unroll
    for (int i = 0; i < 9; ++i) { const float2 v = __ldg(q + i); out[2 * i] = v.x; out[2 * i + 1] = v.y; }
  }
}
// t_e = C_e x for every point, a thread per coupling (couplings of a point are consecutive): each warp stages its 32
// consecutive coupling blocks through shared memory with coalesced 8-byte loads, forms C_c x_r for its coupling, and
// sums the couplings of each point by a segmented scan across the warp; a point that lies inside one warp is stored,
// one split across warps is added atomically into t (zeroed before).
template <class T>
__global__ void __launch_bounds__(256) k_point_ct36(int64_t ncoup, const int32_t* __restrict__ eliminated_ptr,
                                                    const int32_t* __restrict__ entry_eliminated, const int32_t* __restrict__ entry_retained,
                                                    const T* __restrict__ C, const double* __restrict__ x, double* __restrict__ t,
                                                    const Status* __restrict__ st) {
  __shared__ T cs[8][32 * 18];
  if (!live(st)) return;   // uniform
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t cw0 = (blockIdx.x * (int64_t)blockDim.x) + 32 * wid;   // the warp's first coupling
  if (cw0 >= ncoup) return;   // uniform per warp
  const int nw = (int)(ncoup - cw0 < 32 ? ncoup - cw0 : 32);
  // the warp's blocks, in pairs of entries (C is aligned to two entries)
  {
    using V2 = typename std::conditional<std::is_same<T, double>::value, double2, float2>::type;
    const V2* src = reinterpret_cast<const V2*>(C + 18 * cw0);
    V2* dst = reinterpret_cast<V2*>(cs[wid]);
    for (int i = lane; i < 9 * nw; i += 32) dst[i] = __ldg(src + i);
  }
  __syncwarp();
  const int64_t c = cw0 + lane;
  const bool valid = lane < nw;
  int e = valid ? __ldg(entry_eliminated + c) : -1 - lane;   // lanes past the end: segments of their own
  double t0 = 0.0, t1 = 0.0, t2 = 0.0;
  if (valid) {
    const int r = __ldg(entry_retained + c);
    const double2* xp = reinterpret_cast<const double2*>(x + 6 * (int64_t)r);
    const double2 a = __ldg(xp), b = __ldg(xp + 1), d = __ldg(xp + 2);
    const double xr[6] = {a.x, a.y, b.x, b.y, d.x, d.y};
    const T* cb = cs[wid] + 18 * lane;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      t0 += (double)cb[3 * j] * xr[j];
      t1 += (double)cb[3 * j + 1] * xr[j];
      t2 += (double)cb[3 * j + 2] * xr[j];
    }
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double u0 = __shfl_up_sync(0xffffffffu, t0, off), u1 = __shfl_up_sync(0xffffffffu, t1, off),
                 u2 = __shfl_up_sync(0xffffffffu, t2, off);
    const int eu = __shfl_up_sync(0xffffffffu, e, off);
    if (lane >= off && eu == e) {
      t0 += u0;
      t1 += u1;
      t2 += u2;
    }
  }
  const int en = __shfl_down_sync(0xffffffffu, e, 1);
  if (valid && (lane == 31 || en != e)) {   // the last coupling of its point within the warp
    double* te = t + 3 * (int64_t)e;
    if (__ldg(eliminated_ptr + e) >= cw0 && __ldg(eliminated_ptr + e + 1) <= cw0 + nw) {
      te[0] = t0;
      te[1] = t1;
      te[2] = t2;
    } else {
      atomicAdd(te, t0);
      atomicAdd(te + 1, t1);
      atomicAdd(te + 2, t2);
    }
  }
}

// w_e = E^-1 t_e (FP64), a thread per point
__global__ void __launch_bounds__(256) k_point_einv36(int64_t neb, const double* __restrict__ Einv64, const double* __restrict__ t,
                                                      double* __restrict__ w, const Status* __restrict__ st) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb || !live(st)) return;
  const double* inv = Einv64 + 9 * e;
  const double t0 = t[3 * e], t1 = t[3 * e + 1], t2 = t[3 * e + 2];
#pragma unroll
  for (int i = 0; i < 3; ++i) w[3 * e + i] = inv[i] * t0 + inv[i + 3] * t1 + inv[i + 6] * t2;
}

template <class T>
__global__ void __launch_bounds__(256) k_gather_ctw36(int64_t nrb, const int32_t* __restrict__ retained_ptr, const int32_t* __restrict__ retained_entry,
                                                      const int32_t* __restrict__ entry_eliminated, const T* __restrict__ C,
                                                      const double* __restrict__ w, const double* __restrict__ y0, double* __restrict__ y,
                                                      const Status* __restrict__ st) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= nrb || !live(st)) return;
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int q = retained_ptr[r] + lane; q < retained_ptr[r + 1]; q += 32) {
    const int c = __ldg(retained_entry + q), e = __ldg(entry_eliminated + c);
    const double w0 = w[3 * e], w1 = w[3 * e + 1], w2 = w[3 * e + 2];
    T cb[18];
    coupling18<T>(C, c, cb);
#pragma unroll
    for (int j = 0; j < 6; ++j) acc[j] += (double)cb[3 * j] * w0 + (double)cb[3 * j + 1] * w1 + (double)cb[3 * j + 2] * w2;
  }
#pragma unroll
  for (int j = 0; j < 6; ++j)
    for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
  if (lane < 6) {
    double v = 0.0;
#pragma unroll
    for (int j = 0; j < 6; ++j)
      if (j == lane) v = acc[j];
    y[6 * r + lane] = y0[6 * r + lane] - v;
  }
}

// The point term of the reduced operator applied to a vector, in FP64 (no counterpart in the reference, which forms
// S): per eliminated block e, w_e = E_e^-1 sum_c C_c x_r(c), with E^-1 the plan's FP64 inverse of the damped block
// from its last reduction (C_c is d_e x d_r column-major). k_gradient then forms y = y0 - sum_c C_c' w_e(c).
template <class T>
__global__ void __launch_bounds__(256) k_point_apply(int64_t neb, const int32_t* __restrict__ eliminated_ptr,
                                                     const int32_t* __restrict__ entry_retained, const int32_t* __restrict__ e_dims,
                                                     const int32_t* __restrict__ eoffsets, const int32_t* __restrict__ boffsets_e,
                                                     const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boffsets_r,
                                                     const int32_t* __restrict__ coffsets, const T* __restrict__ C,
                                                     const double* __restrict__ Einv64, const double* __restrict__ x,
                                                     double* __restrict__ w, const Status* __restrict__ st) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb || !live(st)) return;
  const int de = e_dims[e];
  double t[3] = {0.0, 0.0, 0.0};
  for (int c = eliminated_ptr[e]; c < eliminated_ptr[e + 1]; ++c) {
    const int r = entry_retained[c], dr = r_dims[r], xo = boffsets_r[r], co = coffsets[c];
    for (int j = 0; j < dr; ++j) {
      const double xj = x[xo + j];
      for (int i = 0; i < de; ++i) t[i] += (double)C[co + i + de * j] * xj;
    }
  }
  const double* inv = Einv64 + eoffsets[e];
  const int so = boffsets_e[e];
  for (int i = 0; i < de; ++i) {
    double a = 0.0;
    for (int k = 0; k < de; ++k) a += inv[i + de * k] * t[k];
    w[so + i] = a;
  }
}

template <class T>
__global__ void __launch_bounds__(128) k_pairs36(
    int64_t nitems, int64_t ncoup, const int32_t* __restrict__ item_block, const int32_t* __restrict__ item_start, const int32_t* __restrict__ item_info,
    const int2* __restrict__ pairs, const int32_t* __restrict__ block_r1, const int32_t* __restrict__ block_r2,
    const int64_t* __restrict__ block_base, const int32_t* __restrict__ block_stride, int64_t dense_nr, const T* __restrict__ C,
    const typename EinvOf<T>::type* __restrict__ Einv12, const double* __restrict__ z, const double* __restrict__ s_r,
    const double* __restrict__ s_e, T* __restrict__ S, double* __restrict__ g, const Status* __restrict__ st,
    const int32_t* __restrict__ prob_of_cam = nullptr, const long long* __restrict__ prob_fail = nullptr) {
  using TE = typename EinvOf<T>::type;
  const int lane = threadIdx.x & 31;
  if (lane >= 30) return;
  const int64_t it = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 5 + lane / 6;
  const int w = lane % 6;
  if (it >= nitems) return;
  if (!live(st)) return;
  const int k = __ldg(item_block + it), pb = __ldg(item_start + it), info = __ldg(item_info + it);
  const int pe = pb + (info & 0xffff);
  const bool solo = (info >> 16) != 0;
  const int r1 = __ldg(block_r1 + k), r2 = __ldg(block_r2 + k);
  if (prob_fail && prob_fail[prob_of_cam[r2]] != NONE) return;   // the block's problem failed: its S stays reset
  const bool diag = r1 == r2;
  const bool scaled = s_r != nullptr || s_e != nullptr;
  const double fw = s_r ? s_r[6 * r2 + w] : 1.0;
  T acc[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) acc[i] = T(0);
  double gacc = 0.0;
  int2 rec = __ldg(pairs + pb);
  for (int p = pb; p < pe; ++p) {
    const int2 cur = rec;
    if (p + 1 < pe) rec = __ldg(pairs + p + 1);
    const int c1 = cur.x, e = cur.y & 0xffffff, c2 = c1 + (cur.y >> 24);
    TE ei[12];
    if constexpr (std::is_same<TE, double>::value) {
      const double2* q = reinterpret_cast<const double2*>(Einv12 + 12 * (int64_t)e);
#pragma unroll
      for (int i = 0; i < 5; ++i) { double2 v = __ldg(q + i); ei[2 * i] = v.x; ei[2 * i + 1] = v.y; }
    } else {
      const float4* q = reinterpret_cast<const float4*>(Einv12 + 12 * (int64_t)e);
#pragma unroll
      for (int i = 0; i < 3; ++i) { float4 v = __ldg(q + i); ei[4 * i] = v.x; ei[4 * i + 1] = v.y; ei[4 * i + 2] = v.z; ei[4 * i + 3] = v.w; }
    }
    T c1v[18];
    if constexpr (std::is_same<T, double>::value) {
      const double2* q = reinterpret_cast<const double2*>(C + 18 * (int64_t)c1);
#pragma unroll
      for (int i = 0; i < 9; ++i) { double2 v = __ldg(q + i); c1v[2 * i] = v.x; c1v[2 * i + 1] = v.y; }
    } else if ((reinterpret_cast<uintptr_t>(C + 18 * (int64_t)c1) & 8) ? c1 > 0 : c1 + 1 < ncoup) {
      // five 16-byte loads from the 16-byte boundary at or below the block (C is 8-byte aligned, so the block starts
      // on a boundary or 8 bytes past one), then its 18 floats at shift 0 or 2. The 20 floats read stay inside C: a
      // shifted read starts in the block before (so not for the first coupling), an unshifted one ends in the block
      // after (so not for the last); those two take the 8-byte path below
      const int sh = (reinterpret_cast<uintptr_t>(C + 18 * (int64_t)c1) & 8) ? 2 : 0;
      const float4* q = reinterpret_cast<const float4*>(C + 18 * (int64_t)c1 - sh);
      float w[20];
#pragma unroll
      for (int i = 0; i < 5; ++i) { float4 v = __ldg(q + i); w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w; }
#pragma unroll
      for (int i = 0; i < 18; ++i) c1v[i] = sh ? w[i + 2] : w[i];
    } else {
      const float2* q = reinterpret_cast<const float2*>(C + 18 * (int64_t)c1);
#pragma unroll
      for (int i = 0; i < 9; ++i) { float2 v = __ldg(q + i); c1v[2 * i] = v.x; c1v[2 * i + 1] = v.y; }
    }
    T c2w[3];
    load_col3(C + 18 * (int64_t)c2 + 3 * w, w & 1, c2w);
    if (scaled) {
      double se[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) se[s] = s_e ? s_e[3 * e + s] : 1.0;
#pragma unroll
      for (int s = 0; s < 3; ++s) c2w[s] = T((double)c2w[s] * (se[s] * fw));
#pragma unroll
      for (int rho = 0; rho < 6; ++rho) {
        const double fr = s_r ? s_r[6 * r1 + rho] : 1.0;
#pragma unroll
        for (int s = 0; s < 3; ++s) c1v[3 * rho + s] = T((double)c1v[3 * rho + s] * (se[s] * fr));
      }
    }
    T u[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) u[t] = (T)(ei[t] * (TE)c2w[0] + ei[t + 3] * (TE)c2w[1] + ei[t + 6] * (TE)c2w[2]);
#pragma unroll
    for (int rho = 0; rho < 6; ++rho) acc[rho] = acc[rho] + c1v[3 * rho] * u[0] + c1v[3 * rho + 1] * u[1] + c1v[3 * rho + 2] * u[2];
    if (diag) {
      const double* zp = z + 3 * (int64_t)e;
      gacc += (double)c2w[0] * zp[0] + (double)c2w[1] * zp[1] + (double)c2w[2] * zp[2];
    }
  }
  const int64_t stride = block_stride ? (int64_t)__ldg(block_stride + k) : dense_nr;
  T* col = S + __ldg(block_base + k) + w * stride;
#pragma unroll
  for (int rho = 0; rho < 6; ++rho) {
    if (diag && rho > w) continue;
    if (solo) col[rho] = col[rho] - acc[rho];
    else atomicAdd(col + rho, -acc[rho]);
  }
  if (diag) {
    if (solo) g[6 * r2 + w] -= gacc;
    else atomicAdd(g + 6 * r2 + w, -gacc);
  }
}

// Add six consecutive entries of a column of S (vector reductions where the address allows: red.global.add.v4/.v2
// for FP32, scalar for FP64). v[i] goes to col[i].
__device__ __forceinline__ void red2(float* p, float a, float b) {
  asm volatile("red.relaxed.gpu.global.add.v2.f32 [%0], {%1, %2};\n" ::"l"(p), "f"(a), "f"(b) : "memory");
}
__device__ __forceinline__ void red4(float* p, float a, float b, float c, float d) {
  asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}
__device__ __forceinline__ void red_column6(float* col, const float v[6]) {
  switch ((reinterpret_cast<uintptr_t>(col) >> 2) & 3) {   // position of col[0] within its 16-byte line
    case 0: red4(col, v[0], v[1], v[2], v[3]); red2(col + 4, v[4], v[5]); break;
    case 1: atomicAdd(col, v[0]); red2(col + 1, v[1], v[2]); red2(col + 3, v[3], v[4]); atomicAdd(col + 5, v[5]); break;
    case 2: red2(col, v[0], v[1]); red4(col + 2, v[2], v[3], v[4], v[5]); break;
    default: atomicAdd(col, v[0]); red4(col + 1, v[1], v[2], v[3], v[4]); atomicAdd(col + 5, v[5]); break;
  }
}
__device__ __forceinline__ void red_column6(double* col, const double v[6]) {
#pragma unroll
  for (int i = 0; i < 6; ++i) atomicAdd(col + i, v[i]);
}

// Phase 2 for d_r = 6, d_e = 3, point-major form: the same pair products as the reference's column-by-column
// accumulation (accumulate_sparse_columns!, src/schur_reduction.jl:315-387), visited by point instead of by S column.
// The pairs (c1, c2), c1 <= c2, of every point, by point, then c2, then c1; six lanes
// per pair (lane w computes column w of C_c1' E^-1 C_c2), five pairs per warp. Consecutive pairs share their point and
// have consecutive c1, so a warp's operands (C of the point's couplings, its padded E^-1) lie in a few contiguous
// lines. Each lane adds its six entries into S with vector reductions (S is expected to stay resident in L2). Record
// {c1, k | (c2 - c1) << 25}: k is the S block (r(c1), r(c2)). The lower triangle of a diagonal block receives -0.0,
// which leaves every value unchanged. Diagonal pairs (c1 = c2, one per coupling) also subtract C_c2' z from g_S.
template <class T>
__global__ void __launch_bounds__(128) k_points36(
    int64_t npairs, const int2* __restrict__ recs, const int32_t* __restrict__ entry_elim, const int32_t* __restrict__ block_r1,
    const int32_t* __restrict__ block_r2, const int64_t* __restrict__ block_base, const int32_t* __restrict__ block_stride,
    int64_t dense_nr, const T* __restrict__ C, const typename EinvOf<T>::type* __restrict__ Einv12, const double* __restrict__ z,
    const double* __restrict__ s_r, const double* __restrict__ s_e, T* __restrict__ S, double* __restrict__ g,
    const Status* __restrict__ st) {
  using TE = typename EinvOf<T>::type;
  const int lane = threadIdx.x & 31;
  if (lane >= 30) return;
  const int64_t q = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 5 + lane / 6;
  const int w = lane % 6;
  if (q >= npairs) return;
  if (!live(st)) return;
  const int2 rec = __ldg(recs + q);
  const uint32_t y = (uint32_t)rec.y;
  const int c1 = rec.x, k = (int)(y & 0x1ffffffu), c2 = c1 + (int)(y >> 25);
  const int e = __ldg(entry_elim + c1);
  const int r1 = __ldg(block_r1 + k), r2 = __ldg(block_r2 + k);
  const bool diag = r1 == r2;
  TE ei[12];
  if constexpr (std::is_same<TE, double>::value) {
    const double2* p = reinterpret_cast<const double2*>(Einv12 + 12 * (int64_t)e);
#pragma unroll
    for (int i = 0; i < 5; ++i) { double2 v = __ldg(p + i); ei[2 * i] = v.x; ei[2 * i + 1] = v.y; }
  } else {
    const float4* p = reinterpret_cast<const float4*>(Einv12 + 12 * (int64_t)e);
#pragma unroll
    for (int i = 0; i < 3; ++i) { float4 v = __ldg(p + i); ei[4 * i] = v.x; ei[4 * i + 1] = v.y; ei[4 * i + 2] = v.z; ei[4 * i + 3] = v.w; }
  }
  T c1v[18];
  if constexpr (std::is_same<T, double>::value) {
    const double2* p = reinterpret_cast<const double2*>(C + 18 * (int64_t)c1);
#pragma unroll
    for (int i = 0; i < 9; ++i) { double2 v = __ldg(p + i); c1v[2 * i] = v.x; c1v[2 * i + 1] = v.y; }
  } else {
    const float2* p = reinterpret_cast<const float2*>(C + 18 * (int64_t)c1);
#pragma unroll
    for (int i = 0; i < 9; ++i) { float2 v = __ldg(p + i); c1v[2 * i] = v.x; c1v[2 * i + 1] = v.y; }
  }
  T c2w[3];
  load_col3(C + 18 * (int64_t)c2 + 3 * w, w & 1, c2w);
  if (s_r != nullptr || s_e != nullptr) {
    const double fw = s_r ? s_r[6 * r2 + w] : 1.0;
    double se[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) se[s] = s_e ? s_e[3 * e + s] : 1.0;
#pragma unroll
    for (int s = 0; s < 3; ++s) c2w[s] = T((double)c2w[s] * (se[s] * fw));
#pragma unroll
    for (int rho = 0; rho < 6; ++rho) {
      const double fr = s_r ? s_r[6 * r1 + rho] : 1.0;
#pragma unroll
      for (int s = 0; s < 3; ++s) c1v[3 * rho + s] = T((double)c1v[3 * rho + s] * (se[s] * fr));
    }
  }
  T u[3];
#pragma unroll
  for (int t = 0; t < 3; ++t) u[t] = (T)(ei[t] * (TE)c2w[0] + ei[t + 3] * (TE)c2w[1] + ei[t + 6] * (TE)c2w[2]);
  T v[6];
#pragma unroll
  for (int rho = 0; rho < 6; ++rho) {
    const T a = c1v[3 * rho] * u[0] + c1v[3 * rho + 1] * u[1] + c1v[3 * rho + 2] * u[2];
    v[rho] = (diag && rho > w) ? T(-0.0) : -a;
  }
  const int64_t stride = block_stride ? (int64_t)__ldg(block_stride + k) : dense_nr;
  red_column6(S + __ldg(block_base + k) + w * stride, v);
  if (diag) {
    const double* zp = z + 3 * (int64_t)e;
    atomicAdd(g + 6 * r2 + w, -((double)c2w[0] * zp[0] + (double)c2w[1] * zp[1] + (double)c2w[2] * zp[2]));
  }
}

// Phase 2 for d_r = 6, d_e = 3, pair-per-lane form with staged operands: one warp per work item (an S block and up
// to 32 of its pairs). The warp first copies the item's operands into shared memory with cp.async, consecutive lanes
// taking consecutive 8-byte chunks of one span (C_c1 and C_c2, 72 bytes each, and the point's padded E^-1), so a copy
// instruction covers a few contiguous spans instead of 32 scattered ones. Then lane i takes pair i whole from shared
// memory (a conflict-free stride of 50 words per pair): U = E^-1 C_c2 (3 x 6) and C_c1' U (the full 6 x 6 block, 108
// FMAs) into 36 register accumulators. The warp sums the lanes' blocks by a reduce-scatter (halving the 36 values over
// lane distances 16 and 8, then a butterfly of the remaining 9 over 4, 2, 1); the lanes with (lane & 7) == 0 write the
// 9 entries of their quarter: plain read-modify-write when the block has a single item, an atomic add otherwise.
// Diagonal items also sum C_c2' z for g_S.
template <class T>
__device__ __forceinline__ T shfl_x(T v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }

template <class T>
__global__ void __launch_bounds__(128) k_pairs_lane(
    int64_t nitems, const int32_t* __restrict__ item_block, const int32_t* __restrict__ item_start, const int32_t* __restrict__ item_info,
    const int2* __restrict__ pairs, const int32_t* __restrict__ block_r1, const int32_t* __restrict__ block_r2,
    const int64_t* __restrict__ block_base, const int32_t* __restrict__ block_stride, int64_t dense_nr, const T* __restrict__ C,
    const typename EinvOf<T>::type* __restrict__ Einv12, const double* __restrict__ z, T* __restrict__ S, double* __restrict__ g,
    const Status* __restrict__ st) {
  using TE = typename EinvOf<T>::type;
  // per pair: C_c1 (18 T), C_c2 (18 T), E^-1 (12 TE), padding; in 8-byte words
  constexpr int WT = (int)sizeof(T) / 4;                     // 4-byte words per T
  constexpr int CW = 18 * WT, EW = 12 * (int)sizeof(TE) / 4;  // words of one C block, of E^-1
  constexpr int PW = 2 * CW + EW + 2;                        // words per pair (50 in FP32, 98 in FP64)
  constexpr int NCH = (2 * CW + EW) / 2;                     // 8-byte chunks per pair
  constexpr int NWARP = sizeof(T) == 4 ? 4 : 3;              // warps per CTA (the FP64 staging is twice as large)
  __shared__ __align__(16) uint32_t stg[NWARP][32 * PW];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t it = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (it >= nitems) return;
  if (!live(st)) return;
  const int k = __ldg(item_block + it), pb = __ldg(item_start + it), info = __ldg(item_info + it);
  const int cnt = info & 0xffff;
  const bool solo = (info >> 16) != 0;
  const int r1 = __ldg(block_r1 + k), r2 = __ldg(block_r2 + k);
  const bool diag = r1 == r2;
  uint32_t* sw = stg[warp];
  int2 mine = make_int2(0, 0);
  if (lane < cnt) mine = __ldg(pairs + pb + lane);
  // chunk q of the item's copies: pair q / NCH (its record fetched from the lane holding it), 8-byte chunk q % NCH
  for (int q0 = 0; q0 < cnt * NCH; q0 += 32) {
    const int q = q0 + lane;
    const int pr = min(q / NCH, 31), sub = q - (q / NCH) * NCH;
    const int c1 = __shfl_sync(0xffffffffu, mine.x, pr), ey = __shfl_sync(0xffffffffu, mine.y, pr);
    if (q < cnt * NCH) {
      const int e = ey & 0xffffff, c2 = c1 + (ey >> 24);
      const char* src;
      if (sub < CW / 2) src = reinterpret_cast<const char*>(C + 18 * (int64_t)c1) + 8 * sub;
      else if (sub < CW) src = reinterpret_cast<const char*>(C + 18 * (int64_t)c2) + 8 * (sub - CW / 2);
      else src = reinterpret_cast<const char*>(Einv12 + 12 * (int64_t)e) + 8 * (sub - CW);
      const unsigned dst = (unsigned)__cvta_generic_to_shared(sw + pr * PW + 2 * sub);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncwarp();
  T acc[36];
#pragma unroll
  for (int i = 0; i < 36; ++i) acc[i] = T(0);
  double gacc[6] = {0, 0, 0, 0, 0, 0};
  if (lane < cnt) {
    const uint32_t* pw = sw + lane * PW;
    T a[18], b[18];
    TE ei[12];
    const T* pa = reinterpret_cast<const T*>(pw);
    const T* pbv = reinterpret_cast<const T*>(pw + CW);
    const TE* pe = reinterpret_cast<const TE*>(pw + 2 * CW);
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        const float2 va = reinterpret_cast<const float2*>(pa)[i], vb = reinterpret_cast<const float2*>(pbv)[i];
        a[2 * i] = va.x; a[2 * i + 1] = va.y; b[2 * i] = vb.x; b[2 * i + 1] = vb.y;
      }
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        const float2 v = reinterpret_cast<const float2*>(pe)[i];
        ei[2 * i] = v.x; ei[2 * i + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 18; ++i) { a[i] = pa[i]; b[i] = pbv[i]; }
#pragma unroll
      for (int i = 0; i < 12; ++i) ei[i] = pe[i];
    }
#pragma unroll
    for (int w = 0; w < 6; ++w) {
      T u[3];
#pragma unroll
      for (int t = 0; t < 3; ++t) u[t] = (T)(ei[t] * (TE)b[3 * w] + ei[t + 3] * (TE)b[3 * w + 1] + ei[t + 6] * (TE)b[3 * w + 2]);
#pragma unroll
      for (int rho = 0; rho < 6; ++rho) acc[6 * w + rho] = acc[6 * w + rho] + a[3 * rho] * u[0] + a[3 * rho + 1] * u[1] + a[3 * rho + 2] * u[2];
    }
    if (diag) {
      const int e = mine.y & 0xffffff;
      const double* zp = z + 3 * (int64_t)e;
      const double z0 = zp[0], z1 = zp[1], z2 = zp[2];
#pragma unroll
      for (int w = 0; w < 6; ++w) gacc[w] = (double)b[3 * w] * z0 + (double)b[3 * w + 1] * z1 + (double)b[3 * w + 2] * z2;
    }
  }
  // reduce-scatter of the 36 accumulators: lanes with bit 4 set keep entries 18..35, then bit 3 splits each half
  T h[18];
  const bool up16 = (lane & 16) != 0;
#pragma unroll
  for (int i = 0; i < 18; ++i) {
    const T send = up16 ? acc[i] : acc[i + 18];
    const T keep = up16 ? acc[i + 18] : acc[i];
    h[i] = keep + shfl_x(send, 16);
  }
  T q9[9];
  const bool up8 = (lane & 8) != 0;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const T send = up8 ? h[i] : h[i + 9];
    const T keep = up8 ? h[i + 9] : h[i];
    q9[i] = keep + shfl_x(send, 8);
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    T v = q9[i];
    v += shfl_x(v, 4);
    v += shfl_x(v, 2);
    v += shfl_x(v, 1);
    q9[i] = v;
  }
  if ((lane & 7) == 0) {
    const int base_idx = (up16 ? 18 : 0) + (up8 ? 9 : 0);
    const int64_t stride = block_stride ? (int64_t)__ldg(block_stride + k) : dense_nr;
    T* blk = S + __ldg(block_base + k);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const int idx = base_idx + i, w = idx / 6, rho = idx - 6 * w;
      if (diag && rho > w) continue;
      T* dst = blk + w * stride + rho;
      if (solo) *dst = *dst - q9[i];
      else atomicAdd(dst, -q9[i]);
    }
  }
  if (diag) {
#pragma unroll
    for (int w = 0; w < 6; ++w) {
      double v = gacc[w];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      gacc[w] = v;
    }
    if (lane < 6) {
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < 6; ++w)
        if (w == lane) v = gacc[w];
      if (solo) g[6 * r2 + lane] -= v;
      else atomicAdd(g + 6 * r2 + lane, -v);
    }
  }
}

// Phase 2 for d_r = 6, d_e = 3 in the canonical layout, owned by block column: one CTA per retained block r2 holds
// the column's S blocks (H x 6, H = col_heights[r2], or the upper part of a dense column) in shared memory and runs the
// column's couplings ("visits": point e seen from r2, the reference's retained_entry order) with a warp per visit. A
// warp stages the point's E^-1 and C_c2 (two contiguous rows of global memory), forms U = E^-1 C_c2 (3 x 6) and the
// gradient term C_c2' z, then lanes (i, rho) take row rho of camera i <= j of the point: the point's coupling blocks
// C_{p0..c2} are contiguous, so a warp's loads cover one contiguous span. Each lane adds its row of C_ci' U to the
// tile with shared-memory atomic adds (visits of different warps may share a block); the tile is written back to S
// once, with no global atomics, and g_S once per column. This is the reference's column-chunk ownership
// (src/schur_reduction.jl:30-49, :362-387) with a warp per coupling entry instead of a thread per column range.
template <class T, bool DENSE>
__global__ void __launch_bounds__(256) k_columns36(
    const int32_t* __restrict__ retained_ptr, const int2* __restrict__ vis_rec, const int32_t* __restrict__ vis_base,
    const uint16_t* __restrict__ vis_off, const int32_t* __restrict__ entry_retained, const int64_t* __restrict__ col_base,
    const int32_t* __restrict__ col_h, int64_t dense_nr, const T* __restrict__ C, const typename EinvOf<T>::type* __restrict__ Einv12,
    const double* __restrict__ z, const double* __restrict__ b_r, const double* __restrict__ s_r, const double* __restrict__ s_e,
    T* __restrict__ S, double* __restrict__ g, const Status* __restrict__ st) {
  using TE = typename EinvOf<T>::type;
  constexpr int NW = 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int r2 = blockIdx.x;
  if (!live(st)) return;
  const int H = DENSE ? 6 * r2 + 6 : __ldg(col_h + r2);
  const int64_t cstride = DENSE ? dense_nr : H;
  const int64_t cb = DENSE ? (int64_t)6 * r2 * dense_nr : __ldg(col_base + r2);
  // shared layout: per-warp staging [NW] { Ei[12] TE | Cj[18] T | U[18] T | zz[4] double }, then the tile [6][H] T
  struct Stage { TE Ei[12]; T Cj[18]; T U[18]; double zz[4]; };
  Stage* stage = reinterpret_cast<Stage*>(smem_raw);
  T* tile = reinterpret_cast<T*>(smem_raw + sizeof(Stage) * NW);
  for (int i = threadIdx.x; i < 6 * H; i += blockDim.x) tile[i] = T(0);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Stage& sg = stage[warp];
  const int q0 = __ldg(retained_ptr + r2), q1 = __ldg(retained_ptr + r2 + 1);
  const int per = (q1 - q0 + NW - 1) / NW;
  const int my0 = min(q1, q0 + warp * per), my1 = min(q1, my0 + per);
  const bool scaled = s_r != nullptr || s_e != nullptr;
  double gacc = 0.0;
  for (int qb = my0; qb < my1; qb += 32) {
    const int q = qb + lane;
    int2 rec = make_int2(0, 0);
    int vbase = 0;
    if (q < my1) { rec = __ldg(vis_rec + q); vbase = __ldg(vis_base + q); }
    const int nv = min(32, my1 - qb);
    for (int v = 0; v < nv; ++v) {
      const int p0 = __shfl_sync(0xffffffffu, rec.x, v);
      const int ey = __shfl_sync(0xffffffffu, rec.y, v);
      const int vb = __shfl_sync(0xffffffffu, vbase, v);
      const int e = ey & 0xffffff, j = ey >> 24, c2 = p0 + j;
      // stage E^-1 (12 lanes), C_c2 (18 lanes) and z (3 lanes): three contiguous rows
      if (lane < 12) sg.Ei[lane] = __ldg(Einv12 + 12 * (int64_t)e + lane);
      else if (lane < 30) {
        const int x = lane - 12;   // x = 3 w + s
        T c = __ldg(C + 18 * (int64_t)c2 + x);
        if (scaled) c = T((double)c * ((s_e ? s_e[3 * e + x % 3] : 1.0) * (s_r ? s_r[6 * r2 + x / 3] : 1.0)));
        sg.Cj[x] = c;
      }
      if (lane < 3) sg.zz[lane] = __ldg(z + 3 * (int64_t)e + lane);
      __syncwarp();
      if (lane < 18) {
        const int t = lane / 6, w = lane % 6;
        sg.U[6 * t + w] = (T)(sg.Ei[t] * (TE)sg.Cj[3 * w] + sg.Ei[t + 3] * (TE)sg.Cj[3 * w + 1] + sg.Ei[t + 6] * (TE)sg.Cj[3 * w + 2]);
      }
      if (lane < 6)
        gacc += (double)sg.Cj[3 * lane] * sg.zz[0] + (double)sg.Cj[3 * lane + 1] * sg.zz[1] + (double)sg.Cj[3 * lane + 2] * sg.zz[2];
      __syncwarp();
      for (int i0 = 0; i0 <= j; i0 += 5) {
        const int i = i0 + lane / 6, rho = lane % 6;
        if (lane < 30 && i <= j) {
          const T* cp = C + 18 * (int64_t)(p0 + i) + 3 * rho;
          T c0 = __ldg(cp), c1 = __ldg(cp + 1), c2v = __ldg(cp + 2);
          const int cam = (DENSE || scaled) ? __ldg(entry_retained + p0 + i) : 0;
          if (scaled) {
            const double fr = s_r ? s_r[6 * cam + rho] : 1.0;
            c0 = T((double)c0 * ((s_e ? s_e[3 * e] : 1.0) * fr));
            c1 = T((double)c1 * ((s_e ? s_e[3 * e + 1] : 1.0) * fr));
            c2v = T((double)c2v * ((s_e ? s_e[3 * e + 2] : 1.0) * fr));
          }
          const int off = DENSE ? 6 * cam : (int)__ldg(vis_off + vb + i);
          T* trow = tile + off + rho;
          const bool diag = i == j;
#pragma unroll
          for (int w = 0; w < 6; ++w) {
            if (diag && rho > w) continue;
            atomicAdd(trow + w * H, c0 * sg.U[w] + c1 * sg.U[6 + w] + c2v * sg.U[12 + w]);
          }
        }
      }
      __syncwarp();
    }
  }
  __shared__ double gpart[NW][6];
  if (lane < 6) gpart[warp][lane] = gacc;
  __syncthreads();
  for (int i = threadIdx.x; i < 6 * H; i += blockDim.x) {
    const int w = i / H, row = i - w * H;
    T* p = S + cb + w * cstride + row;
    *p = *p - tile[i];
  }
  if (threadIdx.x < 6) {
    double a = 0.0;
    for (int w = 0; w < NW; ++w) a += gpart[w][threadIdx.x];
    const int gi = 6 * r2 + threadIdx.x;
    const double bv = s_r ? b_r[gi] * s_r[gi] : b_r[gi];
    g[gi] = bv - a;
  }
}

// Phase 2 for d_r = 6, d_e = 3, sparse S, no conditioning scales: block-column owned and staged in chunks. One CTA
// per retained block r2 holds the column's S blocks (H x 6) in shared memory. Its visits (the points seen from r2, in
// the reference's retained_entry order) are processed in chunks of up to 32: warp 0 sizes a chunk so that the
// visits' coupling spans C_p0 .. C_c2 (contiguous in C) fit the staging buffer, and every warp copies whole spans,
// E^-1 and z into shared memory with cp.async (all of a chunk's loads in flight together). Then each warp takes whole
// visits: lanes 0-17 form U = E^-1 C_c2 (3 x 6) into the warp's slot, lanes 0-5 add C_c2' z to their gradient
// registers, and lanes (i, rho) add row rho of C_i' U to the tile (shared-memory atomic adds: other warps' visits may
// share a block). Two barriers per chunk; S and g_S are written once.
template <class T>
__global__ void __launch_bounds__(256) k_tiles36(
    const int32_t* __restrict__ retained_ptr, const int2* __restrict__ vis_rec, const int32_t* __restrict__ vis_base,
    const uint16_t* __restrict__ vis_off, const int64_t* __restrict__ col_base, const int32_t* __restrict__ col_h, int cap,
    const T* __restrict__ C, const typename EinvOf<T>::type* __restrict__ Einv12, const double* __restrict__ z,
    const double* __restrict__ b_r, T* __restrict__ S, double* __restrict__ g, const Status* __restrict__ st) {
  using TE = typename EinvOf<T>::type;
  constexpr int NV = 32, NW = 8;
  extern __shared__ __align__(16) unsigned char tiles_smem[];
  const int r2 = blockIdx.x;
  if (!live(st)) return;
  const int H = __ldg(col_h + r2);
  const int64_t cb = __ldg(col_base + r2);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned char* ptr = tiles_smem;
  double* zv = reinterpret_cast<double*>(ptr); ptr += sizeof(double) * NV * 3;
  double* gs = reinterpret_cast<double*>(ptr); ptr += sizeof(double) * NW * 6;
  TE* ein = reinterpret_cast<TE*>(ptr); ptr += sizeof(TE) * NV * 12;
  T* U = reinterpret_cast<T*>(ptr); ptr += sizeof(T) * NW * 20;
  int* m_soff = reinterpret_cast<int*>(ptr); ptr += sizeof(int) * NV;
  int* m_j = reinterpret_cast<int*>(ptr); ptr += sizeof(int) * NV;
  int* m_vb = reinterpret_cast<int*>(ptr); ptr += sizeof(int) * NV;
  int* m_p0 = reinterpret_cast<int*>(ptr); ptr += sizeof(int) * NV;
  int* m_e = reinterpret_cast<int*>(ptr); ptr += sizeof(int) * NV;
  int* m_n = reinterpret_cast<int*>(ptr); ptr += sizeof(int) * 4;
  ptr = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(ptr) + 15) & ~uintptr_t(15));
  T* stage = reinterpret_cast<T*>(ptr); ptr += sizeof(T) * cap;
  T* tile = reinterpret_cast<T*>(ptr);
  T* Uw = U + 20 * warp;
  for (int i = tid; i < 6 * H; i += blockDim.x) tile[i] = T(0);
  double gacc = 0.0;   // lanes 0-5: this warp's share of g_S entry 6 r2 + lane
  const int q1 = __ldg(retained_ptr + r2 + 1);
  int q = __ldg(retained_ptr + r2);
  __syncthreads();
  while (q < q1) {
    if (warp == 0) {
      // size the chunk: the longest prefix of the next 32 visits whose spans fit the staging buffer (at least one)
      const int qq = q + lane;
      int2 rec = make_int2(0, 0);
      int vb = 0, sz = 0, j = 0;
      if (qq < q1) {
        rec = __ldg(vis_rec + qq);
        vb = __ldg(vis_base + qq);
        j = rec.y >> 24;
        sz = 18 * (j + 1);
      }
      int ssum = sz;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int a = __shfl_up_sync(0xffffffffu, ssum, o);
        if (lane >= o) ssum += a;
      }
      const bool fits = qq < q1 && (ssum <= cap || lane == 0);
      const int nv = __popc(__ballot_sync(0xffffffffu, fits));
      if (lane < nv) {
        m_soff[lane] = ssum - sz;
        m_j[lane] = j;
        m_vb[lane] = vb;
        m_p0[lane] = rec.x;
        m_e[lane] = rec.y & 0xffffff;
      }
      if (lane == 0) m_n[0] = nv;
    }
    __syncthreads();
    const int nv = m_n[0];
    // stage every visit's span C_p0 .. C_c2, E^-1 and z: a warp per visit, all copies in flight together
    for (int v = warp; v < nv; v += NW) {
      const int n = 18 * (m_j[v] + 1);
      const T* src = C + 18 * (int64_t)m_p0[v];
      T* dst = stage + m_soff[v];
      if (sizeof(T) == 4) {
        for (int x = lane; x < n / 2; x += 32) {
          const unsigned sa = (unsigned)__cvta_generic_to_shared(dst + 2 * x);
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src + 2 * x) : "memory");
        }
      } else {
        for (int x = lane; x < n; x += 32) {
          const unsigned sa = (unsigned)__cvta_generic_to_shared(dst + x);
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src + x) : "memory");
        }
      }
      const int e = m_e[v];
      if (lane < 12) {
        const unsigned sa = (unsigned)__cvta_generic_to_shared(ein + 12 * v + lane);
        if (sizeof(TE) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(Einv12 + 12 * (int64_t)e + lane) : "memory");
        else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(Einv12 + 12 * (int64_t)e + lane) : "memory");
      } else if (lane < 15) {
        const unsigned sa = (unsigned)__cvta_generic_to_shared(zv + 3 * v + (lane - 12));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(z + 3 * (int64_t)e + (lane - 12)) : "memory");
      }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    // a warp per visit
    for (int v = warp; v < nv; v += NW) {
      const int j = m_j[v];
      const T* span = stage + m_soff[v];
      const T* c2 = span + 18 * j;
      if (lane < 18) {
        const int t = lane / 6, w = lane - 6 * t;
        const TE* ei = ein + 12 * v;
        Uw[lane] = (T)(ei[t] * (TE)c2[3 * w] + ei[t + 3] * (TE)c2[3 * w + 1] + ei[t + 6] * (TE)c2[3 * w + 2]);
      }
      if (lane < 6) gacc += (double)c2[3 * lane] * zv[3 * v] + (double)c2[3 * lane + 1] * zv[3 * v + 1] + (double)c2[3 * lane + 2] * zv[3 * v + 2];
      __syncwarp();
      T u[18];
#pragma unroll
      for (int x = 0; x < 18; ++x) u[x] = Uw[x];
      const int vb = m_vb[v], nrow = 6 * (j + 1);
      for (int r = lane; r < nrow; r += 32) {
        const int i = r / 6, rho = r - 6 * i;
        const T* crow = span + 18 * i + 3 * rho;
        const T a0 = crow[0], a1 = crow[1], a2 = crow[2];
        T* trow = tile + (int)__ldg(vis_off + vb + i) + rho;
        const bool diag = i == j;
#pragma unroll
        for (int w = 0; w < 6; ++w) {
          if (diag && rho > w) continue;
          atomicAdd(trow + w * H, a0 * u[w] + a1 * u[6 + w] + a2 * u[12 + w]);
        }
      }
      __syncwarp();
    }
    __syncthreads();
    q += nv;
  }
  if (lane < 6) gs[6 * warp + lane] = gacc;
  __syncthreads();
  for (int i = tid; i < 6 * H; i += blockDim.x) {
    const int w = i / H, row = i - w * H;
    T* p = S + cb + (int64_t)w * H + row;
    *p = *p - tile[i];
  }
  if (tid < 6) {
    double a = 0.0;
    for (int w = 0; w < NW; ++w) a += gs[6 * w + tid];
    g[6 * r2 + tid] = b_r[6 * r2 + tid] - a;
  }
}

// backsubstitute_group! (src/schur_reduction.jl:541-576): x_e = z - E^-1 t, t = sum scaled(C) x_r, all in FP64
template <class T>
__global__ void __launch_bounds__(256) k_backsub(int64_t neb, const int32_t* __restrict__ e_dims, const int32_t* __restrict__ eoffsets,
                                                 const int32_t* __restrict__ boffsets_e, const int32_t* __restrict__ eliminated_ptr,
                                                 const int32_t* __restrict__ entry_retained, const int32_t* __restrict__ coffsets,
                                                 const int32_t* __restrict__ r_dims, const int32_t* __restrict__ boffsets_r,
                                                 const T* __restrict__ C, const double* __restrict__ Einv, const double* __restrict__ z,
                                                 const double* __restrict__ x_r, const double* __restrict__ s_r, const double* __restrict__ s_e,
                                                 double* __restrict__ x_e) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= neb) return;
  const int de = e_dims[e], eo = eoffsets[e], so = boffsets_e[e];
  double t[16] = {};
  for (int c = eliminated_ptr[e]; c < eliminated_ptr[e + 1]; ++c) {
    const int r = entry_retained[c], dr = r_dims[r], ro = boffsets_r[r], co = coffsets[c];
    for (int ir = 0; ir < dr; ++ir) {
      const double xc = x_r[ro + ir], f = s_r ? s_r[ro + ir] : 1.0;
      for (int i = 0; i < de; ++i) {
        T cv = C[co + ir * de + i];
        double cs = (s_r || s_e) ? (double)T((double)cv * ((s_e ? s_e[so + i] : 1.0) * f)) : (double)cv;
        t[i] = t[i] + cs * xc;
      }
    }
  }
  for (int i = 0; i < de; ++i) {
    double acc = Einv[eo + i] * t[0];
    for (int j = 1; j < de; ++j) acc = acc + Einv[eo + i + de * j] * t[j];
    x_e[so + i] = z[so + i] - acc;
  }
}

template <class T>
__global__ void k_gather(T* __restrict__ dest, const T* __restrict__ src, const int64_t* __restrict__ map, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) dest[i] = src[map[i]];
}

// ------------------------------------------------------------------------------------------------------------------
// Plan construction (host, once per structure)
// ------------------------------------------------------------------------------------------------------------------
// Phase 2 for d_r = 6, d_e = 3 and a sparse S, column-owned (the "stage" schedule): one CTA per work item, a run of
// the visits of block column r2 (the points that observe camera r2, in the reference's retained_entry order).
// 1. Each visit's point-side operand W = E' C_c2 (3 x 6, E' = s_e E^-1 s_e from the factor kernel, formed in FP64 and
//    rounded to the storage type) goes to shared memory, with the visit point's first coupling index; the same pass
//    adds C_c2' z' (z' = s_e .* z, FP64) to the column's gradient sums.
// 2. The warps take batches of 32 units, a lane per unit: one S block (r1, r2) and a run of its pairs (c1, c2) of
//    this item, in visit order. The lane owns the whole 6 x 6 block: acc += C_c1' W_c2 (C_c1 from global memory, the
//    next pair's in flight; W_c2 from shared memory), 108 multiply-adds per pair in registers, then the block goes
//    into the column's tile in shared memory (stored when it is its block's only unit, added with atomics otherwise).
//    The diagonal block's pairs (c2, c2) need no batch: step 1 forms C_c2' W of each visit from the operands it holds
//    and stores the sums' upper triangle into the tile's last six rows.
// 3. The tile, times the conditioning scales s_r of its rows and of column r2, is subtracted from the column of S
//    (contiguous: the column's six scalar columns of H entries each), with atomics when the column is split into
//    several items;
//    g_S[r2] -= s_r .* sum C_c2' z'.
// The reference's accumulate_sparse_columns! (src/schur_reduction.jl:315-387) walks the same pairs of each column; W
// is its W_c2 = E^-1 scaled(C_c2) with the point scales folded in, and the pair product C_c1' W_c2 its W_c1' C_c2
// transposed (E^-1 is symmetric).
template <class T>
__host__ __device__ constexpr int stage_wr() { return sizeof(T) == 4 ? 20 : 18; }   // W record stride (16-byte multiple)
// threads per CTA of k_stage36: 256 in FP32 (two CTAs per SM at 128 registers), 128 in FP64 (two per SM at ~240)
template <class T>
__host__ __device__ constexpr int stage_nt() { return sizeof(T) == 4 ? 256 : 128; }
template <class T>
static size_t stage_smem(int64_t max_h, int64_t max_nv) {
  const size_t tile = ((size_t)6 * max_h * sizeof(T) + 15) & ~size_t(15);
  const size_t w = (size_t)max_nv * stage_wr<T>() * sizeof(T);
  const size_t p0 = ((size_t)max_nv * 4 + 15) & ~size_t(15);
  return tile + w + p0 + (stage_nt<T>() / 32) * (6 * sizeof(double) + 21 * sizeof(T));
}

// 18 entries of one coupling block of C, read with 32-byte loads from the 32-byte boundary at or below the block (C on
// a 32-byte boundary): FP32 blocks (72 bytes at 18 c floats) start 0, 2, 4 or 6 floats past a boundary and lie in the
// three 32-byte chunks from it; FP64 blocks (144 bytes) start 0 or 2 doubles past one and lie in five. The last block
// of C takes 8-byte loads instead, so that nothing past C's end is read.
__device__ __forceinline__ void ld256(const float* p, float* w) {
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(w[0]), "=f"(w[1]), "=f"(w[2]), "=f"(w[3]), "=f"(w[4]), "=f"(w[5]), "=f"(w[6]), "=f"(w[7]) : "l"(p));
}
__device__ __forceinline__ void ld256(const double* p, double* w) {
  asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(w[0]), "=d"(w[1]), "=d"(w[2]), "=d"(w[3]) : "l"(p));
}
// The raw chunks of block c (24 floats / 20 doubles) and its shift within them.
struct Raw32 { float w[24]; int sh; };
struct Raw64 { double w[20]; int sh; };
__device__ __forceinline__ void load_raw(const float* __restrict__ C, int64_t c, int64_t ncoup, Raw32& r) {
  const int64_t f = 18 * c;
  r.sh = (int)(f & 7);
  if (c + 1 < ncoup || r.sh == 6) {
    const float* q = C + (f - r.sh);
    ld256(q, r.w);
    ld256(q + 8, r.w + 8);
    ld256(q + 16, r.w + 16);
  } else {
    const float2* q = reinterpret_cast<const float2*>(C + f);
#pragma unroll
    for (int i = 0; i < 9; ++i) { float2 v = __ldg(q + i); r.w[2 * i] = v.x; r.w[2 * i + 1] = v.y; }
    r.sh = 0;
  }
}
__device__ __forceinline__ void load_raw(const double* __restrict__ C, int64_t c, int64_t ncoup, Raw64& r) {
  const int64_t f = 18 * c;
  r.sh = (int)(f & 3);   // 0 or 2
  if (c + 1 < ncoup || r.sh == 2) {
    const double* q = C + (f - r.sh);
#pragma unroll
    for (int i = 0; i < 5; ++i) ld256(q + 4 * i, r.w + 4 * i);
  } else {
    const double2* q = reinterpret_cast<const double2*>(C + f);
#pragma unroll
    for (int i = 0; i < 9; ++i) { double2 v = __ldg(q + i); r.w[2 * i] = v.x; r.w[2 * i + 1] = v.y; }
    r.sh = 0;
  }
}
// the block's 18 entries from its raw chunks (two selects per entry for FP32, one for FP64)
__device__ __forceinline__ void take18(const Raw32& r, float* a) {
  float t[20];
  const bool b4 = (r.sh & 4) != 0, b2 = (r.sh & 2) != 0;
#pragma unroll
  for (int i = 0; i < 20; ++i) t[i] = b4 ? r.w[i + 4] : r.w[i];
#pragma unroll
  for (int i = 0; i < 18; ++i) a[i] = b2 ? t[i + 2] : t[i];
}
__device__ __forceinline__ void take18(const Raw64& r, double* a) {
  const bool b2 = r.sh != 0;
#pragma unroll
  for (int i = 0; i < 18; ++i) a[i] = b2 ? r.w[i + 2] : r.w[i];
}
template <class T> struct RawOf { using type = Raw32; };
template <> struct RawOf<double> { using type = Raw64; };
__device__ __forceinline__ void load_block18(const float* __restrict__ C, int64_t c, int64_t ncoup, float* a) {
  Raw32 r;
  load_raw(C, c, ncoup, r);
  take18(r, a);
}
__device__ __forceinline__ void load_block18(const double* __restrict__ C, int64_t c, int64_t ncoup, double* a) {
  Raw64 r;
  load_raw(C, c, ncoup, r);
  take18(r, a);
}
__device__ __forceinline__ void load_w18(const float* w, float* b) {
  const float4* q = reinterpret_cast<const float4*>(w);
#pragma unroll
  for (int i = 0; i < 4; ++i) { float4 v = q[i]; b[4 * i] = v.x; b[4 * i + 1] = v.y; b[4 * i + 2] = v.z; b[4 * i + 3] = v.w; }
  const float2 v = reinterpret_cast<const float2*>(w)[8];
  b[16] = v.x;
  b[17] = v.y;
}
__device__ __forceinline__ void load_w18(const double* w, double* b) {
  const double2* q = reinterpret_cast<const double2*>(w);
#pragma unroll
  for (int i = 0; i < 9; ++i) { double2 v = q[i]; b[2 * i] = v.x; b[2 * i + 1] = v.y; }
}

template <class T>
__global__ void __launch_bounds__(stage_nt<T>(), 2) k_stage36(
    const int4* __restrict__ items, const int32_t* __restrict__ ibat, const int2* __restrict__ bat, const uint32_t* __restrict__ lane_rec,
    const uint32_t* __restrict__ pairs,
    const int2* __restrict__ vis_rec, const int32_t* __restrict__ col_h, const int64_t* __restrict__ col_base, int64_t ncoup,
    const T* __restrict__ C, const double* __restrict__ EZ, const double* __restrict__ s_r, T* __restrict__ S, double* __restrict__ g,
    const Status* __restrict__ st, const int32_t* __restrict__ prob_of_cam, const long long* __restrict__ prob_fail, int64_t nitems,
    unsigned long long* __restrict__ queue, const int32_t* __restrict__ S_rowval) {
  constexpr int NT = stage_nt<T>();
  constexpr int WR = stage_wr<T>();
  using Raw = typename RawOf<T>::type;
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ int s_item, s_bat;
  if (!live(st)) return;
  const int tid = threadIdx.x, lane = tid & 31;
  // persistent: each CTA takes the next item (in column order) from the queue until none is left
  for (;;) {
  if (tid == 0) {
    s_item = (int)atomicAdd(queue, 1ull);
    s_bat = 0;
  }
  __syncthreads();
  const int item = s_item;
  if (item >= nitems) break;
  const int4 it = items[item];
  const int r2 = it.x, q0 = it.y, nv = it.z, nseg = it.w;
  if (prob_fail && prob_fail[prob_of_cam[r2]] != NONE) {   // the column's problem failed: its S stays reset
    __syncthreads();
    continue;
  }
  const int H = __ldg(col_h + r2);
  T* tile = reinterpret_cast<T*>(sm);
  T* W = reinterpret_cast<T*>(sm + (((size_t)6 * H * sizeof(T) + 15) & ~size_t(15)));
  int* p0s = reinterpret_cast<int*>(W + (size_t)nv * WR);
  double* gp = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(p0s) + (((size_t)nv * 4 + 15) & ~size_t(15)));
  T* dgp = reinterpret_cast<T*>(gp + 6 * (NT / 32));   // per warp, its sums of the diagonal block's upper triangle
  for (int i = tid; i < 6 * H; i += NT) tile[i] = T(0);
  // 1. W, the gradient sums and the diagonal block, a thread per visit ({first coupling, point | index of c2 << 24} per
  //    visit); the next visit's record is loaded while the current one is formed. The diagonal block (c2, c2) takes
  //    C_c2' W of every visit, the product a batch would form, from the operands already in registers: its upper
  //    triangle (dg[c (c + 1) / 2 + rho], rho <= c) is summed per thread, then per warp and over the warps.
  double ga[6];
#pragma unroll
  for (int w = 0; w < 6; ++w) ga[w] = 0.0;
  T dg[21];
#pragma unroll
  for (int i = 0; i < 21; ++i) dg[i] = T(0);
  {
    // FP64 also has the current visit's coupling block in flight from the previous iteration (and the next visit's
    // record from the one before); FP32 has no registers left for it (it would spill)
    constexpr bool PF = sizeof(T) == 8;
    int2 vr = tid < nv ? __ldg(vis_rec + q0 + tid) : make_int2(0, 0);
    int2 vn = make_int2(0, 0);
    Raw rc;
    if constexpr (PF) {
      if (tid + NT < nv) vn = __ldg(vis_rec + q0 + tid + NT);
      if (tid < nv) load_raw(C, vr.x + (int)((unsigned)vr.y >> 24), ncoup, rc);
    }
    for (int v = tid; v < nv; v += NT) {
      const double2* ez = reinterpret_cast<const double2*>(EZ + 12 * (int64_t)(vr.y & 0xffffff));
      double Ep[12];
#pragma unroll
      for (int i = 0; i < 6; ++i) { double2 x = __ldg(ez + i); Ep[2 * i] = x.x; Ep[2 * i + 1] = x.y; }
      T c[18];
      int2 vf = make_int2(0, 0);   // the record fetched in this iteration
      if constexpr (PF) {
        take18(rc, c);
        if (v + NT < nv) load_raw(C, vn.x + (int)((unsigned)vn.y >> 24), ncoup, rc);
        if (v + 2 * NT < nv) vf = __ldg(vis_rec + q0 + v + 2 * NT);
      } else {
        load_block18(C, vr.x + (int)((unsigned)vr.y >> 24), ncoup, c);
        if (v + NT < nv) vf = __ldg(vis_rec + q0 + v + NT);
      }
      p0s[v] = vr.x;
      T* wv = W + (size_t)v * WR;
#pragma unroll
      for (int w = 0; w < 6; ++w) {
        const double c0 = (double)c[3 * w], c1 = (double)c[3 * w + 1], c2v = (double)c[3 * w + 2];
#pragma unroll
        for (int t = 0; t < 3; ++t) wv[3 * w + t] = T(Ep[t] * c0 + Ep[t + 3] * c1 + Ep[t + 6] * c2v);
        ga[w] += c0 * Ep[9] + c1 * Ep[10] + c2v * Ep[11];
      }
      T wr[18];
      load_w18(wv, wr);   // this thread's own W row, back from shared memory (vector loads) rather than held
#pragma unroll
      for (int cc = 0; cc < 6; ++cc)
#pragma unroll
        for (int rho = 0; rho <= cc; ++rho) {
          T x = dg[cc * (cc + 1) / 2 + rho];
          x = fma(c[3 * rho], wr[3 * cc], x);
          x = fma(c[3 * rho + 1], wr[3 * cc + 1], x);
          x = fma(c[3 * rho + 2], wr[3 * cc + 2], x);
          dg[cc * (cc + 1) / 2 + rho] = x;
        }
      if constexpr (PF) {
        vr = vn;
        vn = vf;
      } else {
        vr = vf;
      }
    }
  }
  // the gradient sums, per warp into shared memory (added up after phase 2)
#pragma unroll
  for (int w = 0; w < 6; ++w) {
    double x = ga[w];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) gp[6 * (tid >> 5) + w] = x;
  }
#pragma unroll
  for (int i = 0; i < 21; ++i) {
    T x = dg[i];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) dgp[21 * (tid >> 5) + i] = x;
  }
  __syncthreads();
  // the diagonal block into the tile's last six rows (no batch writes there), the warps' sums in warp order
  if (tid < 21) {
    int cc = 0;
    while ((cc + 1) * (cc + 2) / 2 <= tid) ++cc;
    const int rho = tid - cc * (cc + 1) / 2;
    T x = dgp[tid];
    for (int w = 1; w < NT / 32; ++w) x += dgp[21 * w + tid];
    tile[cc * H + (H - 6) + rho] = x;
  }
  // 2. the item's batches, taken by the warps from a counter, longest first; a lane per unit of the batch
  {
    const int bb = __ldg(ibat + item), nb = __ldg(ibat + item + 1) - bb;
    for (;;) {
      int b = 0;
      if (lane == 0) b = atomicAdd(&s_bat, 1);
      b = __shfl_sync(0xffffffffu, b, 0);
      if (b >= nb) break;
      const int2 br = __ldg(bat + bb + b);   // {first pair, iterations}
      const uint32_t lr = __ldg(lane_rec + (int64_t)(bb + b) * 32 + lane);
      const int len = (int)((lr >> 16) & 0x7fff), iters = br.y;
      const uint32_t* pc = pairs + br.x + lane;
      // the codes of the current and the next iteration; the block of the current one is in flight
      uint32_t cur = __ldg(pc), nxt = iters > 1 ? __ldg(pc + 32) : 0u;
      Raw raw;
      if (len > 0) load_raw(C, p0s[cur & 0xffff] + (int)(cur >> 16), ncoup, raw);
      T acc[36];
#pragma unroll
      for (int i = 0; i < 36; ++i) acc[i] = T(0);
      for (int it = 0; it < iters; ++it) {
        if (it < len) {
          T a[18], w[18];
          take18(raw, a);
          load_w18(W + (size_t)(cur & 0xffff) * WR, w);
          // the next pair's block, in flight during this pair's products
          if (it + 1 < len) load_raw(C, p0s[nxt & 0xffff] + (int)(nxt >> 16), ncoup, raw);
#pragma unroll
          for (int rho = 0; rho < 6; ++rho)
#pragma unroll
            for (int c = 0; c < 6; ++c) {
              T x = acc[6 * rho + c];
              x = fma(a[3 * rho], w[3 * c], x);
              x = fma(a[3 * rho + 1], w[3 * c + 1], x);
              x = fma(a[3 * rho + 2], w[3 * c + 2], x);
              acc[6 * rho + c] = x;
            }
        }
        cur = nxt;
        if (it + 2 < iters) nxt = __ldg(pc + (int64_t)(it + 2) * 32);
      }
      if (len > 0) {
        // the unit's block into the tile: a plain store when it is its block's only unit in the item
        T* tb = tile + (lr & 0xffff);
        if (lr >> 31) {
#pragma unroll
          for (int c = 0; c < 6; ++c)
#pragma unroll
            for (int rho = 0; rho < 6; ++rho) tb[c * H + rho] = acc[6 * rho + c];
        } else {
#pragma unroll
          for (int c = 0; c < 6; ++c)
#pragma unroll
            for (int rho = 0; rho < 6; ++rho) atomicAdd(tb + c * H + rho, acc[6 * rho + c]);
        }
      }
    }
  }
  __syncthreads();
  // 3. the column of S (times the conditioning scales of the tile's rows and of the column) and the gradient
  // a thread per tile row: its conditioning scale once, then the row's six entries (one per scalar column), all six
  // loads of S in flight together
  const int64_t cb = __ldg(col_base + r2);
  double fc[6];
#pragma unroll
  for (int w = 0; w < 6; ++w) fc[w] = s_r ? s_r[6 * r2 + w] : 1.0;
  for (int rr = tid; rr < H; rr += NT) {
    const double f = s_r ? s_r[__ldg(S_rowval + cb + rr)] : 1.0;
    T* Sr = S + cb + rr;
    if (nseg == 1) {
      T old[6];
#pragma unroll
      for (int w = 0; w < 6; ++w) old[w] = Sr[(int64_t)w * H];
#pragma unroll
      for (int w = 0; w < 6; ++w) Sr[(int64_t)w * H] = old[w] - T((double)tile[w * H + rr] * (f * fc[w]));
    } else {
#pragma unroll
      for (int w = 0; w < 6; ++w) atomicAdd(Sr + (int64_t)w * H, -T((double)tile[w * H + rr] * (f * fc[w])));
    }
  }
  if (tid < 6) {
    double x = 0.0;
    for (int w = 0; w < NT / 32; ++w) x += gp[6 * w + tid];
    atomicAdd(g + 6 * r2 + tid, -(s_r ? s_r[6 * r2 + tid] : 1.0) * x);
  }
  __syncthreads();   // the item's shared memory is free for the next one
  }
}

// One column-owned schedule of k_stage36 (SchurPlan::stage[sd], sd 0 for FP32 and 1 for FP64), from the structure:
// each column's pairs grouped by block slot, each block's in visit order. An item is a run of one block column's
// visits: its shared memory holds the column's S tile (6 H entries) and per visit W = E' C_c2 (18 entries) and the
// visit point's first coupling; sized in FP64 bytes this must fit the schedule's STAGE_BUDGET, so a column with more
// visits is cut into several items (their tiles are added to S with atomics). Items stay in column order: neighbouring columns read the couplings of
// overlapping sets of points, which then stay in L2 while the columns in flight move along the cameras.
// A block's pairs of one item are cut into units of at most stage_unit[sd] pairs (the diagonal block's pairs are formed
// by the kernel's staging pass and have no units). The units, longest first,
// are cut into batches of 32 consecutive ones, a lane per unit: the lanes of a batch run units of about the same
// length and write them to the tile at the same time (a warp-wide shared-memory store or atomic costs the same for
// one lane as for 32), and the CTA's warps take batches from a counter in shared memory, longest first, so that they
// finish the item together. Among units of one length the first units of their blocks come first, then the second
// ones, so that the units of one block fall on different lanes. A batch's pairs are stored iteration by iteration, 32
// codes (one per lane) each, so that a warp reads them as one 128-byte line per iteration.
static bool build_stage_schedule(SchurPlan* P, int sd, cudaStream_t s, int64_t nrb, const std::vector<int32_t>& rptr,
                                 const std::vector<int32_t>& rentry, const std::vector<int32_t>& entry_elim, const int64_t* eptr,
                                 const int64_t* eret, const std::vector<int64_t>& bcolptr, const std::vector<int64_t>& browval,
                                 const std::vector<int64_t>& brow_off, const std::vector<int64_t>& col_h) {
  // the shared-memory budget of an item, sized in FP64 bytes (48 per tile row, 148 per visit): 200 KB for the FP32
  // schedule (whose FP32 items then take about 110 KB, two 256-thread CTAs per SM), 96 KB for the FP64 one (two
  // 128-thread CTAs per SM)
  const int64_t STAGE_BUDGET = sd == 0 ? 200 * 1024 : 96 * 1024;
  const int U = P->stage_unit[sd];
  struct ColOut {
    std::vector<int4> items;
    std::vector<int32_t> nbat;   // per item its number of batches
    std::vector<int2> bat;       // batches: first pair relative to the column's `pairs`, iterations
    std::vector<uint32_t> lane, pairs;
    int64_t nunits = 0;
  };
  std::vector<ColOut> out(nrb);
  // one launch serves every item, with the largest column tile and the largest visit run: the visit cap is set by the
  // largest tile, so that any item's share fits the same shared-memory size
  int64_t max_h = 0;
  for (int64_t r2 = 0; r2 < nrb; ++r2) max_h = std::max<int64_t>(max_h, col_h[r2]);
  const int64_t vcap = (STAGE_BUDGET - 48 * max_h - 2048) / 148;
  if (vcap < 32 || max_h > 65535) return false;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(| : bad)
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    const int64_t nv = rptr[r2 + 1] - rptr[r2];
    if (nv == 0) continue;
    const int64_t kb = bcolptr[r2], nbc = bcolptr[r2 + 1] - kb;
    // the kernel adds the diagonal block at rows H - 6 .. H - 1 of the tile: the column's last block must be (r2, r2)
    if (nbc == 0 || browval[kb + nbc - 1] != r2 || brow_off[kb + nbc - 1] != col_h[r2] - 6) {
      bad = 1;
      continue;
    }
    const int64_t nseg = (nv + vcap - 1) / vcap;
    std::vector<int64_t> bnd(nseg + 1);
    for (int64_t g = 0; g <= nseg; ++g) bnd[g] = g * nv / nseg;
    // the column's off-diagonal pairs (c1 < c2 of the points observing r2) in visit order, then grouped by block slot
    // (a counting sort keeps visit order within a block): {visit within its item | c1's index within its point << 16}
    std::vector<int32_t> p_slot, p_seg;
    std::vector<uint32_t> p_code;
    std::vector<int32_t> cnt(nbc + 1, 0);
    for (int64_t g = 0; g < nseg; ++g)
      for (int64_t va = bnd[g]; va < bnd[g + 1]; ++va) {
        const int32_t c2 = rentry[rptr[r2] + va];
        const int64_t e = entry_elim[c2], v = va - bnd[g];
        for (int64_t c1 = eptr[e]; c1 < c2; ++c1) {
          const int64_t* lo = browval.data() + kb;
          const int64_t* f = std::lower_bound(lo, lo + nbc, eret[c1]);
          const int64_t i1 = c1 - eptr[e];
          if (f == lo + nbc || *f != eret[c1] || v > 65535 || i1 > 65535) {
            bad = 1;
            continue;
          }
          p_slot.push_back((int32_t)(f - lo));
          p_seg.push_back((int32_t)g);
          p_code.push_back((uint32_t)v | ((uint32_t)i1 << 16));
          cnt[f - lo + 1] += 1;
        }
      }
    for (int64_t i = 0; i < nbc; ++i) cnt[i + 1] += cnt[i];
    std::vector<int32_t> order(p_slot.size());
    {
      std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
      for (size_t i = 0; i < p_slot.size(); ++i) order[pos[p_slot[i]]++] = (int32_t)i;
    }
    struct Unit { int32_t k, j; bool sole; std::vector<uint32_t> pr; };
    std::vector<std::vector<Unit>> seg_units(nseg);
    for (int64_t sl = 0; sl < nbc; ++sl) {
      int64_t cur = -1;
      std::vector<size_t> first(nseg, SIZE_MAX);   // per segment the block's first unit
      for (int32_t x = cnt[sl]; x < cnt[sl + 1]; ++x) {
        const int32_t i = order[x];
        const int32_t g = p_seg[i];
        if (g != cur || (int)seg_units[g].back().pr.size() == U) {
          if (first[g] == SIZE_MAX) first[g] = seg_units[g].size();
          const int32_t j = (int32_t)(seg_units[g].size() - first[g]);
          seg_units[g].push_back({(int32_t)(kb + sl), j, true, {}});
          cur = g;
        }
        seg_units[g].back().pr.push_back(p_code[i]);
      }
      for (int64_t g = 0; g < nseg; ++g)
        if (first[g] != SIZE_MAX && seg_units[g].size() - first[g] > 1)
          for (size_t i = first[g]; i < seg_units[g].size(); ++i) seg_units[g][i].sole = false;
    }
    ColOut& o = out[r2];
    for (int64_t g = 0; g < nseg; ++g) {
      auto& us = seg_units[g];
      // the off-diagonal units longest first; among units of one length the first units of their blocks, then the
      // second ones, ..., so that the units of one block fall on different lanes (or batches)
      std::stable_sort(us.begin(), us.end(), [](const Unit& x, const Unit& y) {
        return x.pr.size() != y.pr.size() ? x.pr.size() > y.pr.size() : x.j < y.j;
      });
      o.items.push_back(make_int4((int32_t)r2, (int32_t)(rptr[r2] + bnd[g]), (int32_t)(bnd[g + 1] - bnd[g]), (int32_t)nseg));
      o.nbat.push_back((int32_t)((us.size() + 31) / 32));
      o.nunits += (int64_t)us.size();
      // batches of 32 consecutive units: a lane per unit, as many iterations as the batch's first (longest) unit
      for (size_t b0 = 0; b0 < us.size(); b0 += 32) {
        const int32_t iters = (int32_t)us[b0].pr.size();
        o.bat.push_back(make_int2((int32_t)o.pairs.size(), iters));
        for (int L = 0; L < 32; ++L) {
          if (b0 + L < us.size()) {
            const Unit& u = us[b0 + L];
            o.lane.push_back((uint32_t)brow_off[u.k] | ((uint32_t)u.pr.size() << 16) | (u.sole ? 0x80000000u : 0u));
          } else {
            o.lane.push_back(0u);
          }
        }
        for (int32_t it = 0; it < iters; ++it)
          for (int L = 0; L < 32; ++L) {
            const size_t i = b0 + L;
            o.pairs.push_back(i < us.size() && it < (int32_t)us[i].pr.size() ? us[i].pr[it] : 0u);
          }
      }
    }
  }
  if (bad) return false;
  int64_t nitems = 0, nbat = 0, nslots = 0, max_nv = 0, nunits = 0;
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    nitems += (int64_t)out[r2].items.size();
    nbat += (int64_t)out[r2].bat.size();
    nslots += (int64_t)out[r2].pairs.size();
    nunits += out[r2].nunits;
    for (const int4& it : out[r2].items) max_nv = std::max<int64_t>(max_nv, it.z);
  }
  if (nslots >= INT32_MAX || nbat >= INT32_MAX / 32 || nitems >= INT32_MAX) return false;
  std::vector<int4> items;
  std::vector<int32_t> ibat;
  std::vector<int2> bat;
  std::vector<uint32_t> lane, pairs;
  items.reserve(nitems);
  ibat.reserve(nitems + 1);
  bat.reserve(nbat);
  lane.reserve(nbat * 32);
  pairs.reserve(nslots);
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    ColOut& o = out[r2];
    const int32_t pbase = (int32_t)pairs.size();
    int32_t first = (int32_t)bat.size();
    for (int32_t n : o.nbat) {
      ibat.push_back(first);
      first += n;
    }
    items.insert(items.end(), o.items.begin(), o.items.end());
    for (int2 b : o.bat) bat.push_back(make_int2(b.x + pbase, b.y));
    lane.insert(lane.end(), o.lane.begin(), o.lane.end());
    pairs.insert(pairs.end(), o.pairs.begin(), o.pairs.end());
    std::vector<int4>().swap(o.items);
    std::vector<int2>().swap(o.bat);
    std::vector<uint32_t>().swap(o.lane);
    std::vector<uint32_t>().swap(o.pairs);
  }
  ibat.push_back((int32_t)bat.size());
  pairs.resize(pairs.size() + 32, 0u);   // the kernel's read-ahead of the next iteration's codes stays inside the array
  SchurPlan::StageSchedule& S = P->stage[sd];
  upload(S.stg_items, items, s);
  upload(S.stg_ibat, ibat, s);
  upload(S.stg_bat, bat, s);
  upload(S.stg_lane, lane, s);
  upload(S.stg_pairs, pairs, s);
  S.items = nitems;
  S.units = nunits;
  S.batches = nbat;
  S.slots = nslots;
  S.max_nv = max_nv;
  return true;
}

static SchurPlan* plan_create(bls_ctx* ctx, const bls_schur_plan_desc* d) {
  if (!d || d->nrblocks < 1 || d->neblocks < 1) throw Error(BLS_EINVAL, "a plan needs at least one retained and one eliminated block");
  std::unique_ptr<SchurPlan> P(new SchurPlan());
  P->ctx = ctx;
  cudaStream_t s = ctx->stream;
  const int64_t nrb = d->nrblocks, neb = d->neblocks;
  P->nrblocks = nrb;
  P->neblocks = neb;
  const int64_t nc = d->eliminated_ptr[neb];
  P->ncoup = nc;
  std::vector<int64_t> boff_r(nrb), boff_e(neb);
  int64_t nr = 0, ne = 0;
  P->uniform36 = true;
  for (int64_t r = 0; r < nrb; ++r) {
    if (d->r_dims[r] < 1 || d->r_dims[r] > 16) throw Error(BLS_EUNSUPPORTED, "retained block sizes above 16 are not supported on the device");
    boff_r[r] = nr; nr += d->r_dims[r];
    P->max_dr = std::max<int>(P->max_dr, (int)d->r_dims[r]);
    if (d->r_dims[r] != 6) P->uniform36 = false;
  }
  for (int64_t e = 0; e < neb; ++e) {
    if (d->e_dims[e] < 1 || d->e_dims[e] > 16) throw Error(BLS_EUNSUPPORTED, "eliminated block sizes above 16 are not supported on the device");
    boff_e[e] = ne; ne += d->e_dims[e];
    P->max_de = std::max<int>(P->max_de, (int)d->e_dims[e]);
    if (d->e_dims[e] != 3) P->uniform36 = false;
    if (d->eoffsets[e] < 0 || d->eliminated_ptr[e + 1] < d->eliminated_ptr[e]) throw Error(BLS_EINVAL, "malformed structure arrays");
  }
  P->nr = nr;
  P->ne = ne;
  P->E_length = neb ? d->eoffsets[neb - 1] + d->e_dims[neb - 1] * d->e_dims[neb - 1] : 0;
  int64_t clen = 0;
  for (int64_t e = 0; e < neb; ++e)
    for (int64_t c = d->eliminated_ptr[e]; c < d->eliminated_ptr[e + 1]; ++c) {
      const int64_t r = d->entry_retained[c];
      if (r < 0 || r >= nrb) throw Error(BLS_EINVAL, "entry_retained out of range");
      if (c > d->eliminated_ptr[e] && d->entry_retained[c - 1] >= r) throw Error(BLS_EINVAL, "entry_retained must ascend within each eliminated block");
      clen = std::max(clen, d->coffsets[c] + d->r_dims[r] * d->e_dims[e]);
    }
  P->C_length = clen;
  if (clen >= INT32_MAX || P->E_length >= INT32_MAX || nc >= INT32_MAX) throw Error(BLS_EUNSUPPORTED, "block storage beyond 2^31 entries is not supported");
  // workspace index (src/schur_reduction.jl:71-85)
  std::vector<int32_t> entry_elim(nc), rptr(nrb + 1, 0), rentry(nc);
  for (int64_t e = 0; e < neb; ++e)
    for (int64_t c = d->eliminated_ptr[e]; c < d->eliminated_ptr[e + 1]; ++c) { entry_elim[c] = (int32_t)e; rptr[d->entry_retained[c] + 1] += 1; }
  for (int64_t r = 0; r < nrb; ++r) rptr[r + 1] += rptr[r];
  {
    std::vector<int32_t> fill(rptr.begin(), rptr.end() - 1);
    for (int64_t c = 0; c < nc; ++c) rentry[fill[d->entry_retained[c]]++] = (int32_t)c;
  }
  // the S blocks: the given pattern, or the couplings' own block pattern for a dense-only plan
  std::vector<int64_t> bcolptr, browval, brow_off, col_h, Scolptr;
  P->has_sparse = d->block_colptr != nullptr;
  if (P->has_sparse) {
    const int64_t nb = d->block_colptr[nrb];
    bcolptr.assign(d->block_colptr, d->block_colptr + nrb + 1);
    browval.assign(d->block_rowval, d->block_rowval + nb);
    brow_off.assign(d->block_row_offsets, d->block_row_offsets + nb);
    col_h.assign(d->col_heights, d->col_heights + nrb);
    Scolptr.assign(d->S_colptr, d->S_colptr + nr + 1);
    P->nnzS = Scolptr[nr];
  } else {
    Structure st;
    st.nrblocks = nrb; st.neblocks = neb;
    st.r_dims.assign(d->r_dims, d->r_dims + nrb);
    st.e_dims.assign(d->e_dims, d->e_dims + neb);
    std::vector<std::vector<int64_t>> coup(neb);
    for (int64_t e = 0; e < neb; ++e) coup[e].assign(d->entry_retained + d->eliminated_ptr[e], d->entry_retained + d->eliminated_ptr[e + 1]);
    finish_structure(st, coup);
    Pattern pat = build_pattern(st, {});
    bcolptr = pat.block_colptr; browval = pat.block_rowval; brow_off = pat.block_row_offsets; col_h = pat.col_heights; Scolptr = pat.S_colptr;
  }
  const int64_t nb = bcolptr[nrb];
  P->nblocks = nb;
  // Every device write must stay inside S: check the pattern the caller handed in before any kernel uses it.
  if (P->has_sparse) {
    for (int64_t r2 = 0; r2 < nrb; ++r2) {
      if (bcolptr[r2 + 1] < bcolptr[r2]) throw Error(BLS_EINVAL, "block_colptr must be non-decreasing");
      for (int64_t w = 0; w < d->r_dims[r2]; ++w) {
        const int64_t j = boff_r[r2] + w;
        if (Scolptr[j] < 0 || Scolptr[j + 1] - Scolptr[j] != col_h[r2]) throw Error(BLS_EINVAL, "S_colptr does not match col_heights");
      }
      for (int64_t k = bcolptr[r2]; k < bcolptr[r2 + 1]; ++k) {
        const int64_t r1 = browval[k];
        if (r1 < 0 || r1 > r2 || (k > bcolptr[r2] && browval[k - 1] >= r1)) throw Error(BLS_EINVAL, "block_rowval must ascend within each column, upper triangle");
        if (brow_off[k] < 0 || brow_off[k] + d->r_dims[r1] > col_h[r2]) throw Error(BLS_EINVAL, "block_row_offsets exceed the column height");
      }
    }
    const int64_t nnz = Scolptr[nr];
    if (d->diag_inds)
      for (int64_t i = 0; i < nr; ++i)
        if (d->diag_inds[i] < 0 || d->diag_inds[i] >= nnz) throw Error(BLS_EINVAL, "diag_inds out of range");
    if (d->r_to_s_map)
      for (int64_t i = 0; i < d->R_length; ++i)
        if (d->r_to_s_map[i] < -1 || d->r_to_s_map[i] >= nnz) throw Error(BLS_EINVAL, "r_to_s_map out of range");
    if (d->S_rowval)
      for (int64_t q = 0; q < nnz; ++q)
        if (d->S_rowval[q] < 0 || d->S_rowval[q] >= nr) throw Error(BLS_EINVAL, "S_rowval out of range");
  }
  for (int64_t e = 0; e < neb; ++e)
    for (int64_t c = d->eliminated_ptr[e]; c < d->eliminated_ptr[e + 1]; ++c)
      if (d->coffsets[c] < 0) throw Error(BLS_EINVAL, "coffsets out of range");
  std::vector<int32_t> b_r1(nb), b_r2(nb), b_stride(nb);
  std::vector<int64_t> b_base(nb), b_base_dense(nb);
  for (int64_t r2 = 0; r2 < nrb; ++r2)
    for (int64_t k = bcolptr[r2]; k < bcolptr[r2 + 1]; ++k) {
      b_r1[k] = (int32_t)browval[k];
      b_r2[k] = (int32_t)r2;
      b_stride[k] = (int32_t)col_h[r2];
      b_base[k] = Scolptr[boff_r[r2]] + brow_off[k];
      b_base_dense[k] = boff_r[browval[k]] + boff_r[r2] * nr;
    }
  // pair lists per block, cut into items (columns in parallel; each column's pairs keep ascending c2 per block)
  std::vector<int64_t> col_npairs(nrb, 0);
  std::vector<std::vector<int32_t>> col_c1(nrb), col_c2(nrb), col_cnt(nrb);
  int64_t missing = -1;
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    const int64_t kb = bcolptr[r2], ke = bcolptr[r2 + 1], nbc = ke - kb;
    std::vector<int32_t> cnt(nbc + 1, 0);
    std::vector<int32_t> slot_of;   // slot of each pair in visit order
    std::vector<int32_t> pc1, pc2;
    for (int32_t q = rptr[r2]; q < rptr[r2 + 1]; ++q) {
      const int32_t c2 = rentry[q];
      const int64_t e = entry_elim[c2];
      for (int64_t c1 = d->eliminated_ptr[e]; c1 <= c2; ++c1) {
        const int64_t r1 = d->entry_retained[c1];
        const int64_t* lo = browval.data() + kb;
        const int64_t* hi = browval.data() + ke;
        const int64_t* f = std::lower_bound(lo, hi, r1);
        if (f == hi || *f != r1) {
#pragma omp critical
          missing = r1 * nrb + r2;
          continue;
        }
        const int32_t sl = (int32_t)(f - lo);
        slot_of.push_back(sl);
        pc1.push_back((int32_t)c1);
        pc2.push_back(c2);
        cnt[sl + 1] += 1;
      }
    }
    for (int64_t i = 0; i < nbc; ++i) cnt[i + 1] += cnt[i];
    std::vector<int32_t> o1(pc1.size()), o2(pc2.size());
    std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
    for (size_t i = 0; i < pc1.size(); ++i) {
      const int32_t sl = slot_of[i];
      o1[pos[sl]] = pc1[i];
      o2[pos[sl]++] = pc2[i];
    }
    col_c1[r2].swap(o1);
    col_c2[r2].swap(o2);
    col_cnt[r2].swap(cnt);
    col_npairs[r2] = (int64_t)pc1.size();
  }
  if (missing >= 0)
    throw Error(BLS_EPATTERN, "The sparse pattern has no block (" + std::to_string(missing / nrb + 1) + ", " + std::to_string(missing % nrb + 1) + ")");
  int64_t npairs = 0;
  for (int64_t r2 = 0; r2 < nrb; ++r2) npairs += col_npairs[r2];
  if (npairs >= INT32_MAX) throw Error(BLS_EUNSUPPORTED, "more than 2^31 coupling pairs are not supported");
  P->npairs = npairs;
  std::vector<int32_t> pair_c1(npairs), pair_c2(npairs), it_block, it_start, it_info;
  int64_t off = 0;
  for (int64_t r2 = 0; r2 < nrb; ++r2) {
    std::copy(col_c1[r2].begin(), col_c1[r2].end(), pair_c1.begin() + off);
    std::copy(col_c2[r2].begin(), col_c2[r2].end(), pair_c2.begin() + off);
    const auto& cnt = col_cnt[r2];
    for (int64_t sl = 0; sl + 1 < (int64_t)cnt.size(); ++sl) {
      const int32_t a = cnt[sl], b = cnt[sl + 1];
      if (b == a) continue;
      const int nchunk = (b - a + PAIR_CHUNK - 1) / PAIR_CHUNK;
      for (int32_t x = a; x < b; x += PAIR_CHUNK) {
        it_block.push_back((int32_t)(bcolptr[r2] + sl));
        it_start.push_back((int32_t)(off + x));
        it_info.push_back(std::min(PAIR_CHUNK, b - x) | ((nchunk == 1 ? 1 : 0) << 16));
      }
    }
    off += col_npairs[r2];
    std::vector<int32_t>().swap(col_c1[r2]);
    std::vector<int32_t>().swap(col_c2[r2]);
  }
  P->nitems = (int64_t)it_block.size();
  // fast path: uniform 6/3 blocks in the canonical layout, and pairs that pack into {c1, e | (c2 - c1) << 24}
  std::vector<int2> packed;
  if (P->uniform36 && neb < (1 << 24)) {
    bool canon = true;
    for (int64_t e = 0; e < neb && canon; ++e) canon = d->eoffsets[e] == 9 * e;
    for (int64_t c = 0; c < nc && canon; ++c) canon = d->coffsets[c] == 18 * c;
    if (canon) {
      packed.resize(npairs);
      for (int64_t q = 0; q < npairs && canon; ++q) {
        const int32_t c1 = pair_c1[q], c2 = pair_c2[q];
        const int32_t dc = c2 - c1;
        if (dc < 0 || dc > 127) canon = false;
        packed[q] = make_int2(c1, entry_elim[c2] | (dc << 24));
      }
    }
    P->fast36 = canon;
  }
  // column-kernel arrays: visits in the reference's retained_entry order (column by column, ascending coupling)
  std::vector<int2> vrec;
  std::vector<int32_t> vbase;
  std::vector<uint16_t> voff;
  std::vector<int64_t> cbase;
  std::vector<int32_t> ch;
  if (P->fast36) {
    vrec.resize(nc);
    vbase.resize(nc);
    voff.reserve(npairs);
    cbase.resize(nrb);
    ch.resize(nrb);
    for (int64_t r2 = 0; r2 < nrb; ++r2) {
      cbase[r2] = P->has_sparse ? Scolptr[boff_r[r2]] : 0;
      ch[r2] = (int32_t)col_h[r2];
      P->max_col_h = std::max<int64_t>(P->max_col_h, col_h[r2]);
      if (col_h[r2] > 65535) P->fast36 = false;
      for (int32_t q = rptr[r2]; q < rptr[r2 + 1]; ++q) {
        const int32_t c2 = rentry[q];
        const int64_t e = entry_elim[c2], p0 = d->eliminated_ptr[e], j = c2 - p0;
        vrec[q] = make_int2((int32_t)p0, (int32_t)(e | (j << 24)));
        vbase[q] = (int32_t)voff.size();
        for (int64_t i = 0; i <= j; ++i) {
          const int64_t r1 = d->entry_retained[p0 + i];
          const int64_t* lo = browval.data() + bcolptr[r2];
          const int64_t* hi = browval.data() + bcolptr[r2 + 1];
          const int64_t k = std::lower_bound(lo, hi, r1) - browval.data();
          voff.push_back((uint16_t)brow_off[k]);
        }
      }
    }
  }
  // the column-owned schedule (k_stage36), sparse S only
  if (P->fast36 && P->has_sparse) {
    bool ok = true;
    for (int sd = 0; sd < 2 && ok; ++sd)
      ok = build_stage_schedule(P.get(), sd, s, nrb, rptr, rentry, entry_elim, d->eliminated_ptr, d->entry_retained, bcolptr,
                                browval, brow_off, col_h);
    P->stage_ok = ok;
  }
  // staged work items for the host-buffer reduction: stage j holds points [stage_pt[j], stage_pt[j + 1]); a block's
  // pairs ascend in point within its slot, so its pairs of one stage are a contiguous run, cut into items of at most
  // PAIR_CHUNK pairs (solo when the run makes one item)
  std::vector<int32_t> sb_all, ss_all, si_all;
  if (P->fast36 && P->has_sparse) {
    constexpr int K = SchurPlan::kStages;
    std::vector<uint8_t> stage_of(neb);
    P->stage_pt[0] = 0;
    for (int j = 1; j < K; ++j) {
      const int64_t target = nc * j / K;
      P->stage_pt[j] = std::upper_bound(d->eliminated_ptr, d->eliminated_ptr + neb + 1, target) - d->eliminated_ptr - 1;
      P->stage_pt[j] = std::max(P->stage_pt[j], P->stage_pt[j - 1]);
    }
    P->stage_pt[K] = neb;
    for (int j = 0; j <= K; ++j) P->stage_cp[j] = d->eliminated_ptr[P->stage_pt[j]];
    for (int j = 0; j < K; ++j)
      for (int64_t e = P->stage_pt[j]; e < P->stage_pt[j + 1]; ++e) stage_of[e] = (uint8_t)j;
    std::vector<std::vector<int32_t>> tb(K), ts(K), ti(K);
    const int64_t nit = (int64_t)it_block.size();
    for (int64_t i = 0; i < nit;) {
      const int32_t k = it_block[i];
      int64_t i2 = i;
      while (i2 < nit && it_block[i2] == k) ++i2;
      const int64_t a = it_start[i], b = it_start[i2 - 1] + (it_info[i2 - 1] & 0xffff);
      for (int64_t p = a; p < b;) {
        const int j = stage_of[packed[p].y & 0xffffff];
        int64_t q = p + 1;
        while (q < b && stage_of[packed[q].y & 0xffffff] == j) ++q;
        const bool solo = q - p <= PAIR_CHUNK;
        for (int64_t x = p; x < q; x += PAIR_CHUNK) {
          tb[j].push_back(k);
          ts[j].push_back((int32_t)x);
          ti[j].push_back((int32_t)std::min<int64_t>(PAIR_CHUNK, q - x) | ((solo ? 1 : 0) << 16));
        }
        p = q;
      }
      i = i2;
    }
    P->stage_item[0] = 0;
    for (int j = 0; j < K; ++j) {
      sb_all.insert(sb_all.end(), tb[j].begin(), tb[j].end());
      ss_all.insert(ss_all.end(), ts[j].begin(), ts[j].end());
      si_all.insert(si_all.end(), ti[j].begin(), ti[j].end());
      P->stage_item[j + 1] = (int64_t)sb_all.size();
    }
    P->staged = true;
  }
  // uploads
  upload(P->r_dims, to32(d->r_dims, nrb, "r_dims"), s);
  upload(P->boffsets_r, to32(boff_r.data(), nrb, "boffsets_r"), s);
  upload(P->e_dims, to32(d->e_dims, neb, "e_dims"), s);
  upload(P->boffsets_e, to32(boff_e.data(), neb, "boffsets_e"), s);
  upload(P->eoffsets, to32(d->eoffsets, neb, "eoffsets"), s);
  upload(P->eliminated_ptr, to32(d->eliminated_ptr, neb + 1, "eliminated_ptr"), s);
  upload(P->entry_retained, to32(d->entry_retained, nc, "entry_retained"), s);
  upload(P->coffsets, to32(d->coffsets, nc, "coffsets"), s);
  upload(P->entry_eliminated, entry_elim, s);
  upload(P->retained_ptr, rptr, s);
  upload(P->retained_entry, rentry, s);
  upload(P->block_r1, b_r1, s);
  upload(P->block_r2, b_r2, s);
  upload(P->block_stride_sparse, b_stride, s);
  upload(P->block_base_sparse, b_base, s);
  upload(P->block_base_dense, b_base_dense, s);
  if (P->fast36) {
    {
      int64_t kmax = 0;
      for (int64_t e = 0; e < neb; ++e) kmax = std::max<int64_t>(kmax, d->eliminated_ptr[e + 1] - d->eliminated_ptr[e]);
      P->tiles_ok = P->has_sparse && 18 * kmax <= 2048;
    }
    upload(P->vis_rec, vrec, s);
    upload(P->vis_base, vbase, s);
    upload(P->vis_off, voff, s);
    upload(P->col_base, cbase, s);
    upload(P->col_h, ch, s);
    upload(P->pair_packed, packed, s);
    if (P->staged) {
      upload(P->st_block, sb_all, s);
      upload(P->st_start, ss_all, s);
      upload(P->st_info, si_all, s);
    }
  } else {
    upload(P->pair_c1, pair_c1, s);
    upload(P->pair_c2, pair_c2, s);
  }
  upload(P->item_block, it_block, s);
  upload(P->item_start, it_start, s);
  upload(P->item_info, it_info, s);
  if (P->has_sparse) {
    if (d->diag_inds) {
      P->diag_inds_host.assign(d->diag_inds, d->diag_inds + nr);
      upload(P->diag_inds, P->diag_inds_host, s);
    }
    if (d->r_to_s_map && d->R_length > 0) {
      P->R_length = d->R_length;
      std::vector<int64_t> m(d->r_to_s_map, d->r_to_s_map + d->R_length);
      upload(P->r_to_s, m, s);
    }
    if (d->S_rowval) {
      std::vector<int32_t> rv = to32(d->S_rowval, P->nnzS, "S_rowval");
      std::vector<int32_t> cl(P->nnzS);
      for (int64_t j = 0; j < nr; ++j)
        for (int64_t q = Scolptr[j]; q < Scolptr[j + 1]; ++q) cl[q] = (int32_t)j;
      upload(P->S_rowval, rv, s);
      upload(P->S_col, cl, s);
    }
    if (d->diag_inds && P->R_length < INT32_MAX) {
      bool inside = true;
      for (int64_t i = 0; i < nr && inside; ++i) inside = d->diag_inds[i] >= Scolptr[i] && d->diag_inds[i] < Scolptr[i + 1];
      if (inside) {
        std::vector<int32_t> rf(P->nnzS, -1);
        for (int64_t i = 0; i < P->R_length; ++i)
          if (d->r_to_s_map[i] >= 0) rf[d->r_to_s_map[i]] = (int32_t)i;
        upload(P->r_from, rf, s);
        upload(P->S_colptr, Scolptr, s);
        P->reset_fused = true;
      }
    }
  }
  P->Einv64.alloc(sizeof(double) * std::max<int64_t>(P->E_length, 1));
  if (!P->fast36) P->Einv32.alloc(sizeof(float) * std::max<int64_t>(P->E_length, 1));
  P->z.alloc(sizeof(double) * std::max<int64_t>(ne, 1));
  if (P->fast36) P->Einv12.alloc(sizeof(double) * 12 * neb);   // sized for FP64; the FP32 form uses half
  if (P->stage_ok) {
    P->EZ.alloc(sizeof(double) * 12 * neb);
    P->kernel = 5;   // the column-owned schedule is the default where it applies
  }
  P->status.alloc(sizeof(Status));
  Status init{NONE, NONE, NONE, 0};
  BLS_CUDA(cudaMemcpyAsync(P->status.p, &init, sizeof(Status), cudaMemcpyHostToDevice, s));
  BLS_CUDA(cudaMallocHost(&P->host_status, sizeof(Status)));
  BLS_CUDA(cudaStreamSynchronize(s));
  return P.release();
}

static int64_t plan_bytes(const SchurPlan* P) {
  const DevBuf* bufs[] = {&P->r_dims, &P->boffsets_r, &P->e_dims, &P->boffsets_e, &P->eoffsets, &P->eliminated_ptr, &P->entry_retained,
                          &P->coffsets, &P->entry_eliminated, &P->retained_ptr, &P->retained_entry, &P->block_r1, &P->block_r2,
                          &P->block_base_sparse, &P->block_stride_sparse, &P->block_base_dense, &P->pair_c1, &P->pair_c2, &P->pair_packed, &P->pt_rec, &P->Einv12, &P->vis_rec, &P->vis_base, &P->vis_off, &P->col_base, &P->col_h, &P->stage[0].stg_items, &P->stage[0].stg_ibat, &P->stage[0].stg_bat, &P->stage[0].stg_lane, &P->stage[0].stg_pairs, &P->stage[1].stg_items, &P->stage[1].stg_ibat, &P->stage[1].stg_bat, &P->stage[1].stg_lane, &P->stage[1].stg_pairs, &P->EZ,
                          &P->item_block, &P->item_start, &P->item_info, &P->r_to_s, &P->diag_inds, &P->S_rowval, &P->S_col, &P->r_from, &P->S_colptr, &P->st_block, &P->st_start, &P->st_info, &P->h_E, &P->h_C, &P->h_R, &P->h_br, &P->h_be, &P->h_scr, &P->h_sce, &P->h_S, &P->h_g, &P->w_apply, &P->t_apply, &P->acc1,
                          &P->Einv64, &P->Einv32, &P->z, &P->status};
  int64_t b = 0;
  for (auto* x : bufs) b += (int64_t)x->bytes;
  return b;
}

// Read the status word (synchronises) and turn it into the reference's verdict.
static int read_status(SchurPlan* P, int64_t* failed_block) {
  cudaStream_t s = P->ctx->stream;
  BLS_CUDA(cudaMemcpyAsync(P->host_status, P->status.p, sizeof(Status), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  const Status st = *P->host_status;
  if (st.einval_r != NONE || st.einval_e != NONE) {
    const bool r = st.einval_r != NONE;
    set_error(std::string(r ? "scaling_r" : "scaling_e") + " must be finite and non-negative, but entry " +
              std::to_string((r ? st.einval_r : st.einval_e) + 1) + " is not");
    if (failed_block) *failed_block = 0;
    return BLS_EINVAL;
  }
  if (st.failed != NONE) {
    if (failed_block) *failed_block = st.failed + 1;
    return BLS_NOT_PD;
  }
  if (failed_block) *failed_block = 0;
  return BLS_OK;
}

static void check_lambda(double lambda) {
  if (!(std::isfinite(lambda) && lambda >= 0)) throw Error(BLS_EINVAL, "lambda must be finite and non-negative, got " + std::to_string(lambda));
}

static void begin_checked(SchurPlan* P, const double* scaling, int64_t n, int which) {
  cudaStream_t s = P->ctx->stream;
  k_status_begin<<<1, 1, 0, s>>>(P->status.as<Status>(), which);
  P->launches += 1;
  if (n > 0) { k_check_scaling<<<grid_for(n, 256), 256, 0, s>>>(scaling, n, P->status.as<Status>(), which); P->launches += 1; }
  BLS_CUDA(cudaGetLastError());
}

// check_damping of scaling_r: one launch for short vectors, else the clearing launch and a grid-wide check
static void check_scaling_r(SchurPlan* P, const double* sc) {
  if (P->nr <= 16384) {
    k_check_scaling1<<<1, 1024, 0, P->ctx->stream>>>(sc, P->nr, P->status.as<Status>(), 0);
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
  } else {
    begin_checked(P, sc, P->nr, 0);
  }
}

template <class T>
static void reset_sparse(SchurPlan* P, T* S, const T* R, const double* sc, double lambda, const double* s_r) {
  if (!P->has_sparse || !P->diag_inds.p) throw Error(BLS_EINVAL, "the plan was created without a sparse pattern");
  if (P->R_length > 0 && !P->r_to_s.p) throw Error(BLS_EINVAL, "the plan has no r -> s map");
  if (s_r && !P->S_rowval.p) throw Error(BLS_EINVAL, "a conditioning scale needs S_rowval in the plan");
  cudaStream_t s = P->ctx->stream;
  Status* st = P->status.as<Status>();
  if (P->reset_fused) {
    check_scaling_r(P, sc);
    k_reset_columns<T><<<std::max(1, grid_for(P->nr * 32, 256)), 256, 0, s>>>(S, R, P->r_from.as<int32_t>(), P->S_colptr.as<int64_t>(),
                                                               s_r ? P->S_rowval.as<int32_t>() : nullptr, P->diag_inds.as<int64_t>(),
                                                               sc, lambda, s_r, P->nr, st);
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
    return;
  }
  begin_checked(P, sc, P->nr, 0);
  k_fill<T><<<std::min<int64_t>(grid_for(P->nnzS, 256), 148 * 16), 256, 0, s>>>(S, P->nnzS, st);
  if (P->R_length > 0)
    k_scatter_r<T><<<std::min<int64_t>(grid_for(P->R_length, 256), 148 * 16), 256, 0, s>>>(S, R, P->r_to_s.as<int64_t>(), P->R_length, st);
  if (s_r)
    k_scale_sparse<T><<<std::min<int64_t>(grid_for(P->nnzS, 256), 148 * 16), 256, 0, s>>>(S, P->S_rowval.as<int32_t>(), P->S_col.as<int32_t>(), s_r, P->nnzS, st);
  k_damp_diag<T><<<grid_for(P->nr, 256), 256, 0, s>>>(S, P->diag_inds.as<int64_t>(), 0, sc, lambda, s_r, P->nr, st);
  k_reset_done<<<1, 1, 0, s>>>(st);
  P->launches += 3 + (P->R_length > 0 ? 1 : 0) + (s_r ? 1 : 0);
  BLS_CUDA(cudaGetLastError());
}

template <class T>
static void reset_dense(SchurPlan* P, T* S, const T* R, const double* sc, double lambda, const double* s_r) {
  cudaStream_t s = P->ctx->stream;
  Status* st = P->status.as<Status>();
  if (P->nr <= 8192) {
    check_scaling_r(P, sc);
    k_reset_dense_columns<T><<<std::max(1, grid_for(P->nr * 32, 256)), 256, 0, s>>>(S, R, sc, lambda, s_r, P->nr, st);
    P->launches += 1;
    BLS_CUDA(cudaGetLastError());
    return;
  }
  begin_checked(P, sc, P->nr, 0);
  k_copy_scaled_dense<T><<<std::min<int64_t>(grid_for(P->nr * P->nr, 256), 148 * 16), 256, 0, s>>>(S, R, s_r, P->nr, st);
  k_damp_diag<T><<<grid_for(P->nr, 256), 256, 0, s>>>(S, nullptr, P->nr, sc, lambda, s_r, P->nr, st);
  k_reset_done<<<1, 1, 0, s>>>(st);
  P->launches += 3;
  BLS_CUDA(cudaGetLastError());
}

template <class T, int MDE, int MDR>
static void launch_pairs(SchurPlan* P, T* S, bool dense, const T* C, const double* s_r, const double* s_e) {
  using TE = typename EinvOf<T>::type;
  const TE* Einv = std::is_same<T, float>::value ? (const TE*)P->Einv32.p : (const TE*)P->Einv64.p;
  if (P->nitems == 0) return;
  k_pairs<T, MDE, MDR><<<grid_for(P->nitems, 128), 128, 0, P->ctx->stream>>>(
      P->nitems, P->item_block.as<int32_t>(), P->item_start.as<int32_t>(), P->item_info.as<int32_t>(), P->pair_c1.as<int32_t>(),
      P->pair_c2.as<int32_t>(), P->block_r1.as<int32_t>(), P->block_r2.as<int32_t>(),
      dense ? P->block_base_dense.as<int64_t>() : P->block_base_sparse.as<int64_t>(), dense ? nullptr : P->block_stride_sparse.as<int32_t>(),
      P->nr, P->r_dims.as<int32_t>(), P->boffsets_r.as<int32_t>(), P->entry_eliminated.as<int32_t>(), P->e_dims.as<int32_t>(),
      P->boffsets_e.as<int32_t>(), P->eoffsets.as<int32_t>(), P->coffsets.as<int32_t>(), C, Einv, s_r, s_e, S, P->status.as<Status>());
}

// The point-major pair records of k_points36, built from the plan's own lists the first time that schedule is chosen
// (a plan that never uses it keeps no copy): every pair of the block-owned items gets its block, then the pairs are
// ordered by point, c2, c1 as {c1, k | (c2 - c1) << 25}. Synchronises.
static void ensure_points(SchurPlan* P) {
  if (P->points_ok || !P->fast36 || P->nblocks >= (int64_t(1) << 25) || P->npairs == 0) return;
  cudaStream_t s = P->ctx->stream;
  std::vector<int32_t> ib(P->nitems), is(P->nitems), ii(P->nitems);
  std::vector<int2> pk(P->npairs);
  BLS_CUDA(cudaMemcpyAsync(ib.data(), P->item_block.p, sizeof(int32_t) * P->nitems, cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaMemcpyAsync(is.data(), P->item_start.p, sizeof(int32_t) * P->nitems, cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaMemcpyAsync(ii.data(), P->item_info.p, sizeof(int32_t) * P->nitems, cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaMemcpyAsync(pk.data(), P->pair_packed.p, sizeof(int2) * P->npairs, cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  std::vector<int32_t> blk(P->npairs);
  for (int64_t i = 0; i < P->nitems; ++i)
    for (int32_t q = is[i]; q < is[i] + (ii[i] & 0xffff); ++q) blk[q] = ib[i];
  const int64_t neb = P->neblocks;
  std::vector<int64_t> ptr(neb + 1, 0);
  for (int64_t q = 0; q < P->npairs; ++q) ptr[(pk[q].y & 0xffffff) + 1] += 1;
  for (int64_t e = 0; e < neb; ++e) ptr[e + 1] += ptr[e];
  std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
  std::vector<int2> rec(P->npairs);
  for (int64_t q = 0; q < P->npairs; ++q) {
    const int32_t c1 = pk[q].x;
    const uint32_t dc = (uint32_t)pk[q].y >> 24;
    rec[fill[pk[q].y & 0xffffff]++] = make_int2(c1, (int32_t)((uint32_t)blk[q] | (dc << 25)));
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t e = 0; e < neb; ++e)
    std::sort(rec.begin() + ptr[e], rec.begin() + ptr[e + 1], [](const int2& a, const int2& b) {
      const int64_t a2 = a.x + (int64_t)((uint32_t)a.y >> 25), b2 = b.x + (int64_t)((uint32_t)b.y >> 25);
      return a2 != b2 ? a2 < b2 : a.x < b.x;
    });
  upload(P->pt_rec, rec, s);
  BLS_CUDA(cudaStreamSynchronize(s));
  P->points_ok = true;
}

template <class T>
static int reduce(SchurPlan* P, T* S, bool dense, double* g, const double* b_r, const double* b_e, const double* sc_e, double lambda,
                  const T* E, const T* C, const double* s_r, const double* s_e, int64_t* failed_block) {
  if (!dense && !P->has_sparse) throw Error(BLS_EINVAL, "the plan was created without a sparse pattern");
  check_lambda(lambda);
  if (P->fast36 && reinterpret_cast<uintptr_t>(C) % (2 * sizeof(T)) != 0)
    throw Error(BLS_EINVAL, "C_data must be aligned to two elements (the device reads coupling blocks in pairs of entries)");
  cudaStream_t s = P->ctx->stream;
  Status* st = P->status.as<Status>();
  // the column-owned schedule reads C with 16-byte loads (C_data on a 16-byte boundary, as the device allocators give)
  const bool c16 = (reinterpret_cast<uintptr_t>(C) & 31) == 0;   // 32-byte loads of C
  const bool batch = P->nprob > 0 && !dense;
  // a batch runs the column-owned schedule unless the block-owned pair lists are chosen (both keep per-problem failure)
  const bool use_stage = P->fast36 && (P->kernel == 5 || (batch && P->kernel != 1)) && !dense && P->stage_ok && c16 &&
                         (!s_r || P->S_rowval.p);
  const int32_t* poc = batch ? P->prob_of_cam.as<int32_t>() : nullptr;
  long long* pf = batch ? P->prob_fail.as<long long>() : nullptr;
  if (batch) {
    k_prob_arm<<<grid_for(P->nprob, 256), 256, 0, s>>>(pf, P->nprob);
    P->launches += 1;
  }
  if (P->fast36) {
    using TE = typename EinvOf<T>::type;
    k_arm36<<<1, 1, 0, s>>>(st);
    if (P->neblocks > 0)
      k_factor36<T><<<grid_for(P->neblocks, 128), 128, 0, s>>>(0, P->neblocks, E, b_e, sc_e, lambda, s_e, P->Einv64.as<double>(),
                                                             use_stage ? nullptr : P->Einv12.as<TE>(), P->z.as<double>(),
                                                             use_stage ? P->EZ.as<double>() : nullptr,
                                                             batch ? P->prob_of_point.as<int32_t>() : nullptr, pf, st);
  } else {
    begin_checked(P, sc_e, P->ne, 1);
    k_arm<<<1, 1, 0, s>>>(st);
    if (P->neblocks > 0)
      k_factor<T><<<grid_for(P->neblocks, 256), 256, 0, s>>>(P->neblocks, P->e_dims.as<int32_t>(), P->eoffsets.as<int32_t>(),
                                                           P->boffsets_e.as<int32_t>(), E, b_e, sc_e, lambda, s_e, P->Einv64.as<double>(),
                                                           std::is_same<T, float>::value ? P->Einv32.as<float>() : nullptr, P->z.as<double>(), st);
  }
  P->launches += 2;   // k_arm, k_factor
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (P->timing) {
    BLS_CUDA(cudaEventCreate(&ev0));
    BLS_CUDA(cudaEventCreate(&ev1));
  }
  if (use_stage) {
    k_g_init<<<grid_for(P->nr, 256), 256, 0, s>>>(g, b_r, s_r, P->nr, st, poc, pf);
    P->launches += 1;
    const SchurPlan::StageSchedule& SS = P->stage[sizeof(T) == 4 ? 0 : 1];
    if (SS.items > 0) {
      const size_t smem = stage_smem<T>(P->max_col_h, SS.max_nv);
      BLS_CUDA(cudaFuncSetAttribute(k_stage36<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      if (ev0) BLS_CUDA(cudaEventRecord(ev0, s));
      P->launches += 1;
      if (P->stage_grid[sizeof(T) == 4 ? 0 : 1] == 0) {
        int per_sm = 0, nsm = 0, dev = 0;
        BLS_CUDA(cudaGetDevice(&dev));
        BLS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        BLS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage36<T>, stage_nt<T>(), smem));
        P->stage_grid[sizeof(T) == 4 ? 0 : 1] = std::max(1, per_sm) * nsm;
      }
      const int64_t grid = std::min<int64_t>(SS.items, P->stage_grid[sizeof(T) == 4 ? 0 : 1]);
      k_stage36<T><<<(unsigned)grid, stage_nt<T>(), smem, s>>>(
          SS.stg_items.as<int4>(), SS.stg_ibat.as<int32_t>(), SS.stg_bat.as<int2>(), SS.stg_lane.as<uint32_t>(), SS.stg_pairs.as<uint32_t>(),
          P->vis_rec.as<int2>(), P->col_h.as<int32_t>(), P->col_base.as<int64_t>(), P->ncoup, C, P->EZ.as<double>(), s_r, S, g, st,
          poc, pf, SS.items,
          reinterpret_cast<unsigned long long*>(&st->pad), P->S_rowval.as<int32_t>());
      if (ev1) BLS_CUDA(cudaEventRecord(ev1, s));
    }
  } else if (P->fast36 && !batch && P->kernel == 0) {
    using TE = typename EinvOf<T>::type;
    struct StageSz { TE a[12]; T b[18]; T c[18]; double d[4]; };
    const int64_t hmax = dense ? P->nr : P->max_col_h;
    const size_t smem = sizeof(StageSz) * 8 + sizeof(T) * 6 * hmax;
    if (smem > 200 * 1024) throw Error(BLS_EUNSUPPORTED, "a block column of S exceeds the shared-memory tile of this build");
    auto kern = dense ? k_columns36<T, true> : k_columns36<T, false>;
    BLS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (ev0) BLS_CUDA(cudaEventRecord(ev0, s));
    P->launches += 1;
    kern<<<(int)P->nrblocks, 256, smem, s>>>(P->retained_ptr.as<int32_t>(), P->vis_rec.as<int2>(), P->vis_base.as<int32_t>(),
                                              P->vis_off.as<uint16_t>(), P->entry_retained.as<int32_t>(), P->col_base.as<int64_t>(),
                                              P->col_h.as<int32_t>(), P->nr, C, P->Einv12.as<TE>(), P->z.as<double>(), b_r, s_r, s_e, S, g, st);
    if (ev1) BLS_CUDA(cudaEventRecord(ev1, s));
  } else if (P->fast36 && !batch && P->kernel == 3 && !dense && !s_r && !s_e && P->tiles_ok) {
    using TE = typename EinvOf<T>::type;
    const int cap = (int)(sizeof(T) == 4 ? 4096 : 2048);
    const size_t fixed = sizeof(double) * 32 * 3 + sizeof(double) * 8 * 6 + sizeof(TE) * 32 * 12 + sizeof(T) * 8 * 20 + sizeof(int) * (32 * 5 + 4) + 16;
    const size_t smem = fixed + sizeof(T) * cap + sizeof(T) * 6 * P->max_col_h;
    if (smem > 200 * 1024) throw Error(BLS_EUNSUPPORTED, "a block column of S exceeds the shared-memory tile of this build");
    BLS_CUDA(cudaFuncSetAttribute(k_tiles36<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (ev0) BLS_CUDA(cudaEventRecord(ev0, s));
    P->launches += 1;
    k_tiles36<T><<<(int)P->nrblocks, 256, smem, s>>>(P->retained_ptr.as<int32_t>(), P->vis_rec.as<int2>(), P->vis_base.as<int32_t>(),
                                                     P->vis_off.as<uint16_t>(), P->col_base.as<int64_t>(), P->col_h.as<int32_t>(), cap, C,
                                                     P->Einv12.as<TE>(), P->z.as<double>(), b_r, S, g, st);
    if (ev1) BLS_CUDA(cudaEventRecord(ev1, s));
  } else if (P->fast36 && !batch && P->kernel == 2 && !s_r && !s_e) {
    using TE = typename EinvOf<T>::type;
    k_g_init<<<grid_for(P->nr, 256), 256, 0, s>>>(g, b_r, s_r, P->nr, st);
    P->launches += 1;
    if (P->nitems > 0) {
      if (ev0) BLS_CUDA(cudaEventRecord(ev0, s));
      P->launches += 1;
      const int lane_threads = sizeof(T) == 4 ? 128 : 96;
      k_pairs_lane<T><<<grid_for(P->nitems * 32, lane_threads), lane_threads, 0, s>>>(
          P->nitems, P->item_block.as<int32_t>(), P->item_start.as<int32_t>(), P->item_info.as<int32_t>(), P->pair_packed.as<int2>(),
          P->block_r1.as<int32_t>(), P->block_r2.as<int32_t>(), dense ? P->block_base_dense.as<int64_t>() : P->block_base_sparse.as<int64_t>(),
          dense ? nullptr : P->block_stride_sparse.as<int32_t>(), P->nr, C, P->Einv12.as<TE>(), P->z.as<double>(), S, g, st);
      if (ev1) BLS_CUDA(cudaEventRecord(ev1, s));
    }
  } else if (P->fast36 && !batch && P->kernel == 4 && P->points_ok) {
    using TE = typename EinvOf<T>::type;
    k_g_init<<<grid_for(P->nr, 256), 256, 0, s>>>(g, b_r, s_r, P->nr, st);
    P->launches += 1;
    if (P->npairs > 0) {
      const int64_t warps = (P->npairs + 4) / 5;
      if (ev0) BLS_CUDA(cudaEventRecord(ev0, s));
      P->launches += 1;
      k_points36<T><<<grid_for(warps * 32, 128), 128, 0, s>>>(
          P->npairs, P->pt_rec.as<int2>(), P->entry_eliminated.as<int32_t>(), P->block_r1.as<int32_t>(), P->block_r2.as<int32_t>(),
          dense ? P->block_base_dense.as<int64_t>() : P->block_base_sparse.as<int64_t>(), dense ? nullptr : P->block_stride_sparse.as<int32_t>(),
          P->nr, C, P->Einv12.as<TE>(), P->z.as<double>(), s_r, s_e, S, g, st);
      if (ev1) BLS_CUDA(cudaEventRecord(ev1, s));
    }
  } else if (P->fast36) {
    using TE = typename EinvOf<T>::type;
    k_g_init<<<grid_for(P->nr, 256), 256, 0, s>>>(g, b_r, s_r, P->nr, st, poc, pf);
    P->launches += 1;
    if (P->nitems > 0) {
      const int64_t warps = (P->nitems + 4) / 5;
      if (ev0) BLS_CUDA(cudaEventRecord(ev0, s));
      P->launches += 1;
      k_pairs36<T><<<grid_for(warps * 32, 128), 128, 0, s>>>(
          P->nitems, P->ncoup, P->item_block.as<int32_t>(), P->item_start.as<int32_t>(), P->item_info.as<int32_t>(), P->pair_packed.as<int2>(),
          P->block_r1.as<int32_t>(), P->block_r2.as<int32_t>(), dense ? P->block_base_dense.as<int64_t>() : P->block_base_sparse.as<int64_t>(),
          dense ? nullptr : P->block_stride_sparse.as<int32_t>(), P->nr, C, P->Einv12.as<TE>(), P->z.as<double>(), s_r, s_e, S, g, st,
          poc, pf);
      if (ev1) BLS_CUDA(cudaEventRecord(ev1, s));
    }
  } else {
    if (ev0) BLS_CUDA(cudaEventRecord(ev0, s));
    if (P->uniform36) launch_pairs<T, 3, 6>(P, S, dense, C, s_r, s_e);
    else if (P->max_de <= 3) launch_pairs<T, 3, 16>(P, S, dense, C, s_r, s_e);
    else if (P->max_de <= 8) launch_pairs<T, 8, 16>(P, S, dense, C, s_r, s_e);
    else launch_pairs<T, 16, 16>(P, S, dense, C, s_r, s_e);
    if (ev1) BLS_CUDA(cudaEventRecord(ev1, s));
    P->launches += 2;
    k_gradient<T><<<grid_for(P->nrblocks * 32, 256), 256, 0, s>>>(
        P->nrblocks, P->retained_ptr.as<int32_t>(), P->retained_entry.as<int32_t>(), P->entry_eliminated.as<int32_t>(), P->r_dims.as<int32_t>(),
        P->boffsets_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boffsets_e.as<int32_t>(), P->coffsets.as<int32_t>(), C, P->z.as<double>(), b_r,
        s_r, s_e, g, st);
  }
  BLS_CUDA(cudaGetLastError());
  if (ev0 && ev1) P->pair_events.push_back({ev0, ev1});
  else { if (ev0) cudaEventDestroy(ev0); if (ev1) cudaEventDestroy(ev1); }
  P->last_dtype = std::is_same<T, float>::value ? BLS_F32 : BLS_F64;
  if (!failed_block) return BLS_OK;
  return read_status(P, failed_block);
}

// reset_schur_sparse! + reduce_schur_sparse! on host buffers. The copy stream brings in scaling_r, R and b_r, then
// E, b_e and scaling_e, then C stage by stage (few large copies: each copy costs a few microseconds of DMA setup);
// the plan's stream resets S as soon as the first copies land, factors every point block once the point data is in,
// and runs each stage's pair items while the next stage's couplings are still being copied. S and g_S are copied
// back only when the status word is clean.
template <class T>
static int reduce_host_impl(SchurPlan* P, T* S_h, double* g_h, const T* R_h, const double* scr_h, double lambda, const double* br_h,
                            const double* be_h, const double* sce_h, const T* E_h, const T* C_h, int64_t* failed_block) {
  if (!P->staged || !P->reset_fused)
    throw Error(BLS_EUNSUPPORTED, "the host-buffer reduction needs a sparse plan on the 6/3 fast path with diag_inds in their columns");
  if (!S_h || !g_h || !scr_h || !br_h || (P->neblocks > 0 && (!be_h || !sce_h || !E_h || !C_h)) || (P->R_length > 0 && !R_h))
    throw Error(BLS_EINVAL, "a host buffer is NULL");
  check_lambda(lambda);
  constexpr int K = SchurPlan::kStages;
  cudaStream_t s = P->ctx->stream;
  if (!P->copy_stream) {
    BLS_CUDA(cudaStreamCreateWithFlags(&P->copy_stream, cudaStreamNonBlocking));
    BLS_CUDA(cudaEventCreateWithFlags(&P->ev_free, cudaEventDisableTiming));
    BLS_CUDA(cudaEventCreateWithFlags(&P->ev_points, cudaEventDisableTiming));
    for (auto& e : P->ev_in) BLS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (P->h_elem != sizeof(T)) {
    P->h_E.alloc(sizeof(T) * std::max<int64_t>(P->E_length, 1));
    P->h_C.alloc(sizeof(T) * std::max<int64_t>(P->C_length, 2));
    P->h_R.alloc(sizeof(T) * std::max<int64_t>(P->R_length, 1));
    P->h_S.alloc(sizeof(T) * std::max<int64_t>(P->nnzS, 1));
    P->h_br.alloc(sizeof(double) * std::max<int64_t>(P->nr, 1));
    P->h_scr.alloc(sizeof(double) * std::max<int64_t>(P->nr, 1));
    P->h_g.alloc(sizeof(double) * std::max<int64_t>(P->nr, 1));
    P->h_be.alloc(sizeof(double) * std::max<int64_t>(P->ne, 1));
    P->h_sce.alloc(sizeof(double) * std::max<int64_t>(P->ne, 1));
    P->h_elem = sizeof(T);
  }
  cudaStream_t cs = P->copy_stream;
  auto h2d = [&](DevBuf& d, size_t off, const void* src, size_t bytes) {
    if (bytes) BLS_CUDA(cudaMemcpyAsync(static_cast<char*>(d.p) + off, src, bytes, cudaMemcpyHostToDevice, cs));
  };
  // the copies overwrite the device inputs only after all earlier work on the plan's stream
  BLS_CUDA(cudaEventRecord(P->ev_free, s));
  BLS_CUDA(cudaStreamWaitEvent(cs, P->ev_free, 0));
  h2d(P->h_scr, 0, scr_h, sizeof(double) * P->nr);
  h2d(P->h_R, 0, R_h, sizeof(T) * P->R_length);
  h2d(P->h_br, 0, br_h, sizeof(double) * P->nr);
  BLS_CUDA(cudaEventRecord(P->ev_in[0], cs));
  h2d(P->h_E, 0, E_h, sizeof(T) * 9 * P->neblocks);
  h2d(P->h_be, 0, be_h, sizeof(double) * P->ne);
  h2d(P->h_sce, 0, sce_h, sizeof(double) * P->ne);
  BLS_CUDA(cudaEventRecord(P->ev_points, cs));
  for (int j = 0; j < K; ++j) {
    const int64_t c0 = P->stage_cp[j], c1 = P->stage_cp[j + 1];
    h2d(P->h_C, sizeof(T) * 18 * c0, C_h + 18 * c0, sizeof(T) * 18 * (c1 - c0));
    BLS_CUDA(cudaEventRecord(P->ev_in[j + 1], cs));
  }
  T* S = P->h_S.as<T>();
  double* g = P->h_g.as<double>();
  Status* st = P->status.as<Status>();
  const bool batch = P->nprob > 0;
  const int32_t* poc = batch ? P->prob_of_cam.as<int32_t>() : nullptr;
  long long* pf = batch ? P->prob_fail.as<long long>() : nullptr;
  BLS_CUDA(cudaStreamWaitEvent(s, P->ev_in[0], 0));
  reset_sparse<T>(P, S, P->h_R.as<T>(), P->h_scr.as<double>(), lambda, nullptr);
  k_arm36<<<1, 1, 0, s>>>(st);
  P->launches += 1;
  if (batch) {
    k_prob_arm<<<grid_for(P->nprob, 256), 256, 0, s>>>(pf, P->nprob);
    P->launches += 1;
  } else {
    k_g_init<<<std::max(1, grid_for(P->nr, 256)), 256, 0, s>>>(g, P->h_br.as<double>(), nullptr, P->nr, st);
    P->launches += 1;
  }
  using TE = typename EinvOf<T>::type;
  BLS_CUDA(cudaStreamWaitEvent(s, P->ev_points, 0));
  if (P->neblocks > 0) {
    k_factor36<T><<<grid_for(P->neblocks, 128), 128, 0, s>>>(0, P->neblocks, P->h_E.as<T>(), P->h_be.as<double>(), P->h_sce.as<double>(), lambda,
                                                             nullptr, P->Einv64.as<double>(), P->Einv12.as<TE>(), P->z.as<double>(), nullptr,
                                                             batch ? P->prob_of_point.as<int32_t>() : nullptr, pf, st);
    P->launches += 1;
  }
  if (batch) {   // after the factorisation: a failing problem keeps its g_S
    k_g_init<<<std::max(1, grid_for(P->nr, 256)), 256, 0, s>>>(g, P->h_br.as<double>(), nullptr, P->nr, st, poc, pf);
    P->launches += 1;
  }
  for (int j = 0; j < K; ++j) {
    BLS_CUDA(cudaStreamWaitEvent(s, P->ev_in[j + 1], 0));
    const int64_t i0 = P->stage_item[j], n = P->stage_item[j + 1] - i0;
    if (n > 0) {
      k_pairs36<T><<<grid_for((n + 4) / 5 * 32, 128), 128, 0, s>>>(
          n, P->ncoup, P->st_block.as<int32_t>() + i0, P->st_start.as<int32_t>() + i0, P->st_info.as<int32_t>() + i0, P->pair_packed.as<int2>(),
          P->block_r1.as<int32_t>(), P->block_r2.as<int32_t>(), P->block_base_sparse.as<int64_t>(), P->block_stride_sparse.as<int32_t>(), P->nr,
          P->h_C.as<T>(), P->Einv12.as<TE>(), P->z.as<double>(), nullptr, nullptr, S, g, st, poc, pf);
      P->launches += 1;
    }
  }
  BLS_CUDA(cudaGetLastError());
  const int rc = read_status(P, failed_block);
  if (rc != BLS_OK) return rc;
  if (batch) {
    // only the problems that succeeded are copied back: a failing problem's S and g_S stay as the caller had them
    std::vector<long long> f((size_t)P->nprob);
    BLS_CUDA(cudaMemcpyAsync(f.data(), pf, sizeof(long long) * P->nprob, cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    for (int64_t a = 0; a < P->nprob;) {
      if (f[a] != NONE) { ++a; continue; }
      int64_t b = a;
      while (b < P->nprob && f[b] == NONE) ++b;   // a run of problems that succeeded: one copy of S and one of g_S
      const int64_t s0 = P->prob_nnz_off[a], s1 = P->prob_nnz_off[b], g0 = P->prob_row_off[a], g1 = P->prob_row_off[b];
      BLS_CUDA(cudaMemcpyAsync(S_h + s0, S + s0, sizeof(T) * (s1 - s0), cudaMemcpyDeviceToHost, s));
      BLS_CUDA(cudaMemcpyAsync(g_h + g0, g + g0, sizeof(double) * (g1 - g0), cudaMemcpyDeviceToHost, s));
      a = b;
    }
  } else {
    BLS_CUDA(cudaMemcpyAsync(S_h, S, sizeof(T) * P->nnzS, cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaMemcpyAsync(g_h, g, sizeof(double) * P->nr, cudaMemcpyDeviceToHost, s));
  }
  BLS_CUDA(cudaStreamSynchronize(s));
  return BLS_OK;
}

// The host call returns only when nothing it enqueued still reads or writes the caller's host buffers: on an error the
// copy stream and the plan's stream are drained before the error is passed on.
template <class T>
static int reduce_host(SchurPlan* P, T* S_h, double* g_h, const T* R_h, const double* scr_h, double lambda, const double* br_h,
                       const double* be_h, const double* sce_h, const T* E_h, const T* C_h, int64_t* failed_block) {
  try {
    return reduce_host_impl<T>(P, S_h, g_h, R_h, scr_h, lambda, br_h, be_h, sce_h, E_h, C_h, failed_block);
  } catch (...) {
    if (P->copy_stream) cudaStreamSynchronize(P->copy_stream);
    cudaStreamSynchronize(P->ctx->stream);
    throw;
  }
}


template <class T>
static double hessian_bilinear(SchurPlan* P, const T* R, bool dense, const T* E, const T* C, const double* x, const double* y) {
  if (!dense && !(P->has_sparse && P->S_rowval.p)) throw Error(BLS_EINVAL, "a sparse R needs a plan with the pattern and S_rowval");
  if (!R || !x || !y || (P->neblocks > 0 && (!E || !C))) throw Error(BLS_EINVAL, "a device pointer is NULL");
  cudaStream_t s = P->ctx->stream;
  if (!P->acc1.p) P->acc1.alloc(sizeof(double));
  double* out = P->acc1.as<double>();
  BLS_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
  const int64_t n = dense ? P->nr * P->nr : P->nnzS;
  k_bilinear_R<T><<<std::max(1, (int)std::min<int64_t>(grid_for(n, 256), 148 * 8)), 256, 0, s>>>(
      P->nnzS, dense ? P->nr : 0, P->S_rowval.as<int32_t>(), P->S_col.as<int32_t>(), R, x, y, out);
  if (P->neblocks > 0)
    k_bilinear_points<T><<<grid_for(P->neblocks, 256), 256, 0, s>>>(
        P->neblocks, P->nr, P->eliminated_ptr.as<int32_t>(), P->entry_retained.as<int32_t>(), P->e_dims.as<int32_t>(), P->eoffsets.as<int32_t>(),
        P->boffsets_e.as<int32_t>(), P->r_dims.as<int32_t>(), P->boffsets_r.as<int32_t>(), P->coffsets.as<int32_t>(), E, C, x, y, out);
  P->launches += 2;
  double h = 0.0;
  BLS_CUDA(cudaMemcpyAsync(&h, out, sizeof(double), cudaMemcpyDeviceToHost, s));
  BLS_CUDA(cudaStreamSynchronize(s));
  return h;
}

template <class T>
static void hessian_diagonal(SchurPlan* P, const T* R, bool dense, const T* E, double* d) {
  if (!dense && !(P->has_sparse && P->diag_inds.p)) throw Error(BLS_EINVAL, "a sparse R needs a plan with the pattern");
  if (!R || !d || (P->neblocks > 0 && !E)) throw Error(BLS_EINVAL, "a device pointer is NULL");
  const int64_t n = std::max(P->nr, P->neblocks);
  k_hessian_diag<T><<<std::max(1, grid_for(n, 256)), 256, 0, P->ctx->stream>>>(P->nr, P->neblocks, P->diag_inds.as<int64_t>(), dense ? P->nr : 0,
                                                                             P->e_dims.as<int32_t>(), P->eoffsets.as<int32_t>(),
                                                                             P->boffsets_e.as<int32_t>(), R, E, d);
  P->launches += 1;
  BLS_CUDA(cudaGetLastError());
}

// y = y0 - C' E^-1 C x over every eliminated block, in FP64, from the plan's E^-1 of its last successful reduction
template <class T>
static int apply_elimination(SchurPlan* P, double* y, const double* y0, const double* x, const T* C) {
  if (P->max_de > 3) throw Error(BLS_EUNSUPPORTED, "the reduced operator is applied for eliminated blocks of size <= 3");
  if (!y || !y0 || !x || (P->ncoup > 0 && !C)) throw Error(BLS_EINVAL, "a device pointer is NULL");
  cudaStream_t s = P->ctx->stream;
  if (!P->w_apply.p) P->w_apply.alloc(sizeof(double) * std::max<int64_t>(P->ne, 1));
  Status* st = P->status.as<Status>();
  if (P->fast36) {
    if (reinterpret_cast<uintptr_t>(C) % (2 * sizeof(T)) != 0)
      throw Error(BLS_EINVAL, "C_data must be aligned to two elements (the device reads coupling blocks in pairs of entries)");
    if (reinterpret_cast<uintptr_t>(x) % 16 != 0) throw Error(BLS_EINVAL, "x must be 16-byte aligned");
    if (P->neblocks > 0) {
      if (!P->t_apply.p) P->t_apply.alloc(sizeof(double) * 3 * (size_t)P->neblocks);
      BLS_CUDA(cudaMemsetAsync(P->t_apply.p, 0, sizeof(double) * 3 * (size_t)P->neblocks, s));
      k_point_ct36<T><<<grid_for(P->ncoup, 256), 256, 0, s>>>(P->ncoup, P->eliminated_ptr.as<int32_t>(), P->entry_eliminated.as<int32_t>(),
                                                              P->entry_retained.as<int32_t>(), C, x, P->t_apply.as<double>(), st);
      k_point_einv36<<<grid_for(P->neblocks, 256), 256, 0, s>>>(P->neblocks, P->Einv64.as<double>(), P->t_apply.as<double>(),
                                                                 P->w_apply.as<double>(), st);
      P->launches += 1;
    }
    if (P->nrblocks > 0)
      k_gather_ctw36<T><<<grid_for(P->nrblocks * 32, 256), 256, 0, s>>>(P->nrblocks, P->retained_ptr.as<int32_t>(), P->retained_entry.as<int32_t>(),
                                                                        P->entry_eliminated.as<int32_t>(), C, P->w_apply.as<double>(), y0, y, st);
    P->launches += 2;
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  }
  if (P->neblocks > 0)
    k_point_apply<T><<<grid_for(P->neblocks, 256), 256, 0, s>>>(
        P->neblocks, P->eliminated_ptr.as<int32_t>(), P->entry_retained.as<int32_t>(), P->e_dims.as<int32_t>(), P->eoffsets.as<int32_t>(),
        P->boffsets_e.as<int32_t>(), P->r_dims.as<int32_t>(), P->boffsets_r.as<int32_t>(), P->coffsets.as<int32_t>(), C,
        P->Einv64.as<double>(), x, P->w_apply.as<double>(), st);
  if (P->nrblocks > 0)
    k_gradient<T><<<grid_for(P->nrblocks * 32, 256), 256, 0, s>>>(
        P->nrblocks, P->retained_ptr.as<int32_t>(), P->retained_entry.as<int32_t>(), P->entry_eliminated.as<int32_t>(), P->r_dims.as<int32_t>(),
        P->boffsets_r.as<int32_t>(), P->e_dims.as<int32_t>(), P->boffsets_e.as<int32_t>(), P->coffsets.as<int32_t>(), C,
        P->w_apply.as<double>(), y0, nullptr, nullptr, y, st);
  P->launches += 2;
  BLS_CUDA(cudaGetLastError());
  return BLS_OK;
}

template <class T>
static void backsub(SchurPlan* P, double* x_e, const double* x_r, const T* C, const double* s_r, const double* s_e) {
  if (P->neblocks == 0) return;
  P->launches += 1;
  k_backsub<T><<<grid_for(P->neblocks, 256), 256, 0, P->ctx->stream>>>(
      P->neblocks, P->e_dims.as<int32_t>(), P->eoffsets.as<int32_t>(), P->boffsets_e.as<int32_t>(), P->eliminated_ptr.as<int32_t>(),
      P->entry_retained.as<int32_t>(), P->coffsets.as<int32_t>(), P->r_dims.as<int32_t>(), P->boffsets_r.as<int32_t>(), C,
      P->Einv64.as<double>(), P->z.as<double>(), x_r, s_r, s_e, x_e);
  BLS_CUDA(cudaGetLastError());
}

}  // namespace bls

// ======================================================================================================================
// C ABI
// ======================================================================================================================
struct bls_schur_plan : bls::SchurPlan {};

using namespace bls;

#define BLS_GUARD(...)                                                        \
  try {                                                                       \
    __VA_ARGS__                                                               \
  } catch (const bls::Error& e) {                                             \
    bls::set_error(e.what());                                                 \
    return e.code;                                                            \
  } catch (const std::bad_alloc&) {                                           \
    bls::set_error("out of host memory");                                     \
    return BLS_ENOMEM;                                                        \
  } catch (const std::exception& e) {                                         \
    bls::set_error(e.what());                                                 \
    return BLS_EINVAL;                                                        \
  }

namespace bls {

// symmetrifyfull! blocks, a warp per block: each lane copies entries of the block and, off the diagonal, their
// transposes (no two blocks write the same entry: the host keeps one of (r, c) and (c, r))
template <class T>
__global__ void __launch_bounds__(256) k_symmetrify(const T* __restrict__ data, const SymBlock* __restrict__ blk, int64_t nblk,
                                                    T* __restrict__ mat, int64_t m) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nblk; t += nwarps) {
    const SymBlock b = blk[t];
    const int sz = b.rd * b.cd;
    for (int q = lane; q < sz; q += 32) {
      const int row = q % b.rd, col = q / b.rd;
      const T v = data[b.src + q];
      mat[(b.rs + row) + m * (b.cs + col)] = v;
      if (!b.diag) mat[(b.cs + col) + m * (b.rs + row)] = v;
    }
  }
}

void launch_symmetrify(cudaStream_t s, int dtype, const void* data, const SymBlock* blocks_host, int64_t nblocks, void* mat,
                       int64_t m) {
  const size_t es = dtype == BLS_F64 ? sizeof(double) : sizeof(float);
  if (m > 0) BLS_CUDA(cudaMemsetAsync(mat, 0, es * (size_t)m * (size_t)m, s));
  if (nblocks == 0) return;
  SymBlock* d = nullptr;
  BLS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(SymBlock) * (size_t)nblocks, s));
  // the stream-ordered block list is released on every path, an error included (freed in stream order after the
  // work queued before it)
  struct FreeAsync {
    SymBlock* p;
    cudaStream_t s;
    ~FreeAsync() { if (p) cudaFreeAsync(p, s); }
  } guard{d, s};
  // from pageable host memory: the list is staged before the call returns
  BLS_CUDA(cudaMemcpyAsync(d, blocks_host, sizeof(SymBlock) * (size_t)nblocks, cudaMemcpyHostToDevice, s));
  const unsigned grid = (unsigned)std::min<int64_t>((nblocks * 32 + 255) / 256, 148 * 16);
  if (dtype == BLS_F64) k_symmetrify<double><<<grid, 256, 0, s>>>((const double*)data, d, nblocks, (double*)mat, m);
  else k_symmetrify<float><<<grid, 256, 0, s>>>((const float*)data, d, nblocks, (float*)mat, m);
  BLS_CUDA(cudaGetLastError());
}

}  // namespace bls

extern "C" {

int bls_schur_plan_create(bls_ctx* ctx, const bls_schur_plan_desc* desc, bls_schur_plan** out) {
  BLS_GUARD({
    if (!ctx || !out) throw Error(BLS_EINVAL, "null argument");
    BLS_CUDA(cudaSetDevice(ctx->device));
    *out = static_cast<bls_schur_plan*>(plan_create(ctx, desc));
    return BLS_OK;
  })
}

int bls_schur_plan_destroy(bls_schur_plan* plan) {
  if (plan) {
    cudaStreamSynchronize(plan->ctx->stream);
    delete static_cast<SchurPlan*>(plan);
  }
  return BLS_OK;
}

int64_t bls_schur_plan_device_bytes(const bls_schur_plan* plan) { return plan ? plan_bytes(plan) : 0; }

int bls_reset_schur_sparse(bls_schur_plan* P, int dtype, void* S, const void* R, const double* sc, double lambda, const double* s_r) {
  BLS_GUARD({
    check_lambda(lambda);
    if (dtype == BLS_F64) reset_sparse<double>(P, (double*)S, (const double*)R, sc, lambda, s_r);
    else if (dtype == BLS_F32) reset_sparse<float>(P, (float*)S, (const float*)R, sc, lambda, s_r);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_reset_schur_dense(bls_schur_plan* P, int dtype, void* S, const void* R, const double* sc, double lambda, const double* s_r) {
  BLS_GUARD({
    check_lambda(lambda);
    if (dtype == BLS_F64) reset_dense<double>(P, (double*)S, (const double*)R, sc, lambda, s_r);
    else if (dtype == BLS_F32) reset_dense<float>(P, (float*)S, (const float*)R, sc, lambda, s_r);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_reduce_schur_sparse(bls_schur_plan* P, int dtype, void* S, double* g, const double* b_r, const double* b_e, const double* sc_e,
                            double lambda, const void* E, const void* C, const double* s_r, const double* s_e, int64_t* failed_block) {
  BLS_GUARD({
    if (dtype == BLS_F64) return reduce<double>(P, (double*)S, false, g, b_r, b_e, sc_e, lambda, (const double*)E, (const double*)C, s_r, s_e, failed_block);
    if (dtype == BLS_F32) return reduce<float>(P, (float*)S, false, g, b_r, b_e, sc_e, lambda, (const float*)E, (const float*)C, s_r, s_e, failed_block);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_hessian_bilinear(bls_schur_plan* P, int dtype, const void* R, int dense, const void* E, const void* C, const double* x,
                         const double* y, double* result) {
  BLS_GUARD({
    if (!P || !result) throw Error(BLS_EINVAL, "null argument");
    if (dtype == BLS_F64) *result = hessian_bilinear<double>(P, (const double*)R, dense != 0, (const double*)E, (const double*)C, x, y);
    else if (dtype == BLS_F32) *result = hessian_bilinear<float>(P, (const float*)R, dense != 0, (const float*)E, (const float*)C, x, y);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_hessian_diagonal(bls_schur_plan* P, int dtype, const void* R, int dense, const void* E, double* d) {
  BLS_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (dtype == BLS_F64) hessian_diagonal<double>(P, (const double*)R, dense != 0, (const double*)E, d);
    else if (dtype == BLS_F32) hessian_diagonal<float>(P, (const float*)R, dense != 0, (const float*)E, d);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_schur_apply_elimination(bls_schur_plan* P, int dtype, double* y, const double* y0, const double* x, const void* C) {
  BLS_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (dtype == BLS_F64) return apply_elimination<double>(P, y, y0, x, (const double*)C);
    if (dtype == BLS_F32) return apply_elimination<float>(P, y, y0, x, (const float*)C);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_reset_reduce_schur_sparse_host(bls_schur_plan* P, int dtype, void* S, double* g, const void* R, const double* sc_r, double lambda,
                                       const double* b_r, const double* b_e, const double* sc_e, const void* E, const void* C,
                                       int64_t* failed_block) {
  BLS_GUARD({
    if (!P) throw Error(BLS_EINVAL, "plan is NULL");
    if (dtype == BLS_F64)
      return reduce_host<double>(P, (double*)S, g, (const double*)R, sc_r, lambda, b_r, b_e, sc_e, (const double*)E, (const double*)C, failed_block);
    if (dtype == BLS_F32)
      return reduce_host<float>(P, (float*)S, g, (const float*)R, sc_r, lambda, b_r, b_e, sc_e, (const float*)E, (const float*)C, failed_block);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_reduce_schur_dense(bls_schur_plan* P, int dtype, void* S, double* g, const double* b_r, const double* b_e, const double* sc_e,
                           double lambda, const void* E, const void* C, const double* s_r, const double* s_e, int64_t* failed_block) {
  BLS_GUARD({
    if (dtype == BLS_F64) return reduce<double>(P, (double*)S, true, g, b_r, b_e, sc_e, lambda, (const double*)E, (const double*)C, s_r, s_e, failed_block);
    if (dtype == BLS_F32) return reduce<float>(P, (float*)S, true, g, b_r, b_e, sc_e, lambda, (const float*)E, (const float*)C, s_r, s_e, failed_block);
    throw Error(BLS_EINVAL, "unknown dtype");
  })
}

int bls_schur_plan_set_kernel(bls_schur_plan* P, int which) {
  if (!P || which < 0 || which > 5) return BLS_EINVAL;
  BLS_GUARD({
    if (which == 4) ensure_points(P);
    P->kernel = which;
    return BLS_OK;
  })
}

// Rebuild the column-owned schedule with units of at most `unit` pairs, from the plan's device copies of the structure
// (the schedule is a plan-time product; this is the autotuner's knob). On failure the previous schedule stays.
int bls_schur_plan_set_stage_unit(bls_schur_plan* P, int unit) {
  if (!P || unit < 1 || unit > 4096) return BLS_EINVAL;
  BLS_GUARD({
    if (!P->fast36 || !P->has_sparse || !P->stage_ok) throw Error(BLS_EUNSUPPORTED, "the plan has no column-owned schedule");
    if (unit == P->stage_unit[0] && unit == P->stage_unit[1]) return BLS_OK;
    cudaStream_t s = P->ctx->stream;
    const int64_t nrb = P->nrblocks, neb = P->neblocks, nc = P->ncoup;
    const int64_t nb = P->nblocks;
    auto down32 = [&](const DevBuf& b, int64_t n) {
      std::vector<int32_t> v((size_t)n);
      if (n) BLS_CUDA(cudaMemcpyAsync(v.data(), b.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      return v;
    };
    std::vector<int32_t> rptr = down32(P->retained_ptr, nrb + 1), rentry = down32(P->retained_entry, nc);
    std::vector<int32_t> entry_elim = down32(P->entry_eliminated, nc), ep32 = down32(P->eliminated_ptr, neb + 1);
    std::vector<int32_t> er32 = down32(P->entry_retained, nc), b_r1 = down32(P->block_r1, nb), b_r2 = down32(P->block_r2, nb);
    std::vector<int32_t> ch = down32(P->col_h, nrb);
    std::vector<int64_t> b_base((size_t)nb), cbase((size_t)nrb);
    if (nb) BLS_CUDA(cudaMemcpyAsync(b_base.data(), P->block_base_sparse.p, (size_t)nb * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaMemcpyAsync(cbase.data(), P->col_base.p, (size_t)nrb * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> eptr(ep32.begin(), ep32.end()), eret(er32.begin(), er32.end());
    std::vector<int64_t> bcolptr(nrb + 1, 0), browval(nb), brow_off(nb), col_h(ch.begin(), ch.end());
    for (int64_t k = 0; k < nb; ++k) {
      bcolptr[b_r2[k] + 1] += 1;
      browval[k] = b_r1[k];
      brow_off[k] = b_base[k] - cbase[b_r2[k]];
    }
    for (int64_t r = 0; r < nrb; ++r) bcolptr[r + 1] += bcolptr[r];
    const int old0 = P->stage_unit[0], old1 = P->stage_unit[1];
    P->stage_unit[0] = P->stage_unit[1] = unit;
    // each schedule is replaced only when its rebuild succeeds (a schedule with the old unit size stays valid)
    bool ok = true;
    for (int sd = 0; sd < 2; ++sd)
      ok = build_stage_schedule(P, sd, s, nrb, rptr, rentry, entry_elim, eptr.data(), eret.data(), bcolptr, browval, brow_off,
                                col_h) && ok;
    if (!ok) {
      P->stage_unit[0] = old0;
      P->stage_unit[1] = old1;
      throw Error(BLS_EUNSUPPORTED, "the schedule does not fit this unit size");
    }
    P->stage_grid[0] = P->stage_grid[1] = 0;
    return BLS_OK;
  })
}

// The phase-2 kernel the next reduction of this storage type launches (the dispatch of reduce(), without the calls).
int bls_schur_plan_phase2_kernel(bls_schur_plan* P, int dtype, int dense, int scaled, char* buf, int64_t cap) {
  if (!P || !buf || cap < 1 || (dtype != BLS_F64 && dtype != BLS_F32)) return BLS_EINVAL;
  const std::string t = dtype == BLS_F32 ? "<float>" : "<double>";
  std::string name;
  if (P->fast36 && (P->kernel == 5 || (P->nprob > 0 && P->kernel != 1)) && !dense && P->stage_ok) name = "k_stage36" + t;
  else if (P->fast36 && P->nprob > 0 && !dense) name = "k_pairs36" + t;
  else if (P->fast36 && P->kernel == 0) name = std::string("k_columns36") + t;
  else if (P->fast36 && P->kernel == 3 && !dense && !scaled && P->tiles_ok) name = "k_tiles36" + t;
  else if (P->fast36 && P->kernel == 2 && !scaled) name = "k_pairs_lane" + t;
  else if (P->fast36 && P->kernel == 4 && P->points_ok) name = "k_points36" + t;
  else if (P->fast36) name = "k_pairs36" + t;
  else name = "k_pairs" + t;
  std::snprintf(buf, (size_t)cap, "%s", name.c_str());
  return BLS_OK;
}

int bls_schur_plan_set_problems(bls_schur_plan* P, int64_t nprob, const int64_t* point_off, const int64_t* camera_off,
                                const int64_t* row_off, const int64_t* nnz_off) {
  BLS_GUARD({
    if (!P) throw Error(BLS_EINVAL, "null plan");
    if (nprob == 0) { P->nprob = 0; return BLS_OK; }
    if (nprob < 0 || !point_off || !camera_off || !row_off || !nnz_off) throw Error(BLS_EINVAL, "null argument");
    if (!P->fast36 || !P->has_sparse)
      throw Error(BLS_EUNSUPPORTED, "per-problem failure needs a sparse plan on the 6/3 fast path");
    if (point_off[0] != 0 || point_off[nprob] != P->neblocks || camera_off[0] != 0 || camera_off[nprob] != P->nrblocks ||
        row_off[0] != 0 || row_off[nprob] != P->nr || nnz_off[0] != 0 || nnz_off[nprob] != P->nnzS)
      throw Error(BLS_EINVAL, "problem offsets must start at 0 and end at the plan's sizes");
    std::vector<int32_t> pop((size_t)P->neblocks), poc((size_t)P->nrblocks);
    for (int64_t p = 0; p < nprob; ++p) {
      if (point_off[p + 1] < point_off[p] || camera_off[p + 1] < camera_off[p] || row_off[p + 1] < row_off[p] || nnz_off[p + 1] < nnz_off[p])
        throw Error(BLS_EINVAL, "problem offsets must be non-decreasing");
      for (int64_t e = point_off[p]; e < point_off[p + 1]; ++e) pop[e] = (int32_t)p;
      for (int64_t r = camera_off[p]; r < camera_off[p + 1]; ++r) poc[r] = (int32_t)p;
    }
    cudaStream_t s = P->ctx->stream;
    upload(P->prob_of_point, pop, s);
    upload(P->prob_of_cam, poc, s);
    P->prob_fail.alloc(sizeof(long long) * (size_t)nprob);
    std::vector<long long> none((size_t)nprob, NONE);
    BLS_CUDA(cudaMemcpyAsync(P->prob_fail.p, none.data(), sizeof(long long) * nprob, cudaMemcpyHostToDevice, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    P->prob_point_off.assign(point_off, point_off + nprob + 1);
    P->prob_row_off.assign(row_off, row_off + nprob + 1);
    P->prob_nnz_off.assign(nnz_off, nnz_off + nprob + 1);
    P->nprob = nprob;
    return BLS_OK;
  })
}

int bls_schur_plan_problem_status(bls_schur_plan* P, int64_t* failed_blocks) {
  BLS_GUARD({
    if (!P || !failed_blocks) throw Error(BLS_EINVAL, "null argument");
    if (P->nprob == 0) throw Error(BLS_EINVAL, "the plan has no problem partition");
    std::vector<long long> f((size_t)P->nprob);
    cudaStream_t s = P->ctx->stream;
    BLS_CUDA(cudaMemcpyAsync(f.data(), P->prob_fail.p, sizeof(long long) * P->nprob, cudaMemcpyDeviceToHost, s));
    BLS_CUDA(cudaStreamSynchronize(s));
    int64_t nfail = 0;
    for (int64_t p = 0; p < P->nprob; ++p) {
      failed_blocks[p] = f[p] == NONE ? 0 : f[p] - P->prob_point_off[p] + 1;
      nfail += f[p] != NONE;
    }
    return nfail ? BLS_NOT_PD : BLS_OK;
  })
}

int bls_schur_plan_instrument(bls_schur_plan* P, int timing) {
  if (!P) return BLS_EINVAL;
  P->timing = timing != 0;
  return BLS_OK;
}

int bls_schur_plan_counters(bls_schur_plan* P, int64_t* launches, double* pair_kernel_ms, int64_t* pair_kernel_launches) {
  BLS_GUARD({
    if (!P) throw Error(BLS_EINVAL, "null plan");
    double ms = 0.0;
    if (!P->pair_events.empty()) BLS_CUDA(cudaEventSynchronize(P->pair_events.back().second));
    for (auto& e : P->pair_events) {
      float t = 0.f;
      BLS_CUDA(cudaEventElapsedTime(&t, e.first, e.second));
      ms += t;
    }
    if (launches) *launches = P->launches;
    if (pair_kernel_ms) *pair_kernel_ms = ms;
    if (pair_kernel_launches) *pair_kernel_launches = (int64_t)P->pair_events.size();
    for (auto& e : P->pair_events) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    P->pair_events.clear();
    P->launches = 0;
    return BLS_OK;
  })
}

int bls_schur_query_status(bls_schur_plan* P, int64_t* failed_block) {
  BLS_GUARD({ return read_status(P, failed_block); })
}

int bls_backsubstitute(bls_schur_plan* P, int dtype, double* x_e, const double* x_r, const void* C, const double* s_r, const double* s_e) {
  BLS_GUARD({
    if (dtype == BLS_F64) backsub<double>(P, x_e, x_r, (const double*)C, s_r, s_e);
    else if (dtype == BLS_F32) backsub<float>(P, x_e, x_r, (const float*)C, s_r, s_e);
    else throw Error(BLS_EINVAL, "unknown dtype");
    return BLS_OK;
  })
}

int bls_scatter_copy(bls_ctx* ctx, int dtype, void* dest, const void* src, const int64_t* map, int64_t n) {
  BLS_GUARD({
    if (n <= 0) return BLS_OK;
    const int grid = (int)std::min<int64_t>(grid_for(n, 256), 148 * 16);
    if (dtype == BLS_F64) k_gather<double><<<grid, 256, 0, ctx->stream>>>((double*)dest, (const double*)src, map, n);
    else if (dtype == BLS_F32) k_gather<float><<<grid, 256, 0, ctx->stream>>>((float*)dest, (const float*)src, map, n);
    else throw Error(BLS_EINVAL, "unknown dtype");
    BLS_CUDA(cudaGetLastError());
    return BLS_OK;
  })
}

}  // extern "C"

