// Seeded synthetic bundle-adjustment scenes, and their assembly into the reference's storage layout.
//
// The workloads name no public dataset; these generators produce scenes with the stated shapes and distributions:
// cameras (block size 6) and points (block size 3), each point observed by k distinct cameras, one row block of 2 rows
// per observation with a 2x6 camera Jacobian, a 2x3 point Jacobian and a 2-vector residual.
//   covisibility "uniform":  k ~ U{kmin..kmax}, cameras drawn without replacement from all cameras;
//   covisibility "window":   centre camera ~ U, k = min(2 + Geometric(p), cap, window size), cameras drawn without
//                            replacement from [centre - w, centre + w] clipped to the camera range;
//   point conditioning:      the stacked 2k x 3 point Jacobian is Q diag(sigma) V' with Q, V Haar-random orthonormal
//                            (Gram-Schmidt of Gaussians) and sigma log-uniform in [sv_lo, sv_hi];
//   camera scales:           each camera's 6 Jacobian columns scaled by log-uniform factors in [cs_lo, cs_hi].
// Random numbers: splitmix64 seeding xoshiro256**, one stream per point (seeded by the point's index), so a scene does
// not depend on the number of threads that generate it. Normals by the Marsaglia polar method.
//
// Assembly follows addblock! (src/schur_assembly.jl:140-246): E += Jp'Jp, C (d_e x d_r, column-major) += Jp'Jc,
// the camera's diagonal block of R += Jc'Jc, b_e += Jp'r, b_r += Jc'r.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

namespace {

inline uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Xoshiro {
  uint64_t s[4];
  explicit Xoshiro(uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {   // xoshiro256**
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }                 // [0, 1)
  double uniform_open() { return ((double)(next() >> 11) + 0.5) * 0x1.0p-53; }    // (0, 1)
  int64_t below(int64_t n) { return (int64_t)(uniform() * (double)n); }
  double normal() {
    for (;;) {
      double u = 2.0 * uniform() - 1.0, v = 2.0 * uniform() - 1.0, q = u * u + v * v;
      if (q > 0.0 && q < 1.0) return u * std::sqrt(-2.0 * std::log(q) / q);
    }
  }
  double loguniform(double lo, double hi) { return std::exp(std::log(lo) + (std::log(hi) - std::log(lo)) * uniform()); }
};

// Columns of A (m x n, column-major) made orthonormal by modified Gram-Schmidt
void orthonormalize(double* A, int m, int n) {
  for (int j = 0; j < n; ++j) {
    double* a = A + (size_t)j * m;
    for (int i = 0; i < j; ++i) {
      const double* q = A + (size_t)i * m;
      double d = 0;
      for (int r = 0; r < m; ++r) d += q[r] * a[r];
      for (int r = 0; r < m; ++r) a[r] -= d * q[r];
    }
    double nrm = 0;
    for (int r = 0; r < m; ++r) nrm += a[r] * a[r];
    nrm = std::sqrt(nrm);
    for (int r = 0; r < m; ++r) a[r] /= nrm;
  }
}

}  // namespace

struct bls_scene {
  int64_t ncams = 0, npoints = 0, nobs = 0;
  std::vector<int64_t> obs_ptr;     // per point, its observations obs_ptr[p] .. obs_ptr[p+1]
  std::vector<int64_t> obs_cam;     // camera of each observation (ascending within a point)
  std::vector<double> Jc, Jp, r;    // per observation: 2x6, 2x3 (column-major), 2
};

extern "C" {

// covis: 0 = uniform, 1 = window. sv_lo <= 0 disables point conditioning; cs_lo <= 0 disables camera scales.
int bls_scene_generate(int64_t ncams, int64_t npoints, int covis, int64_t kmin, int64_t kmax, double geom_p, int64_t kcap,
                       int64_t window, double sv_lo, double sv_hi, double cs_lo, double cs_hi, uint64_t seed, bls_scene** out) {
  if (ncams < 1 || npoints < 1 || !out) return -1;
  auto* S = new bls_scene();
  S->ncams = ncams;
  S->npoints = npoints;
  std::vector<int64_t> k(npoints);
  std::vector<std::vector<int64_t>> cams(npoints);
  // camera column scales
  std::vector<double> cscale;
  if (cs_lo > 0) {
    cscale.resize(ncams * 6);
    Xoshiro rc(seed ^ 0x5ca1ab1e5ca1ab1eull);
    for (auto& x : cscale) x = rc.loguniform(cs_lo, cs_hi);
  }
#pragma omp parallel for schedule(static, 1024)
  for (int64_t p = 0; p < npoints; ++p) {
    uint64_t sd = seed * 0x9E3779B97F4A7C15ull + (uint64_t)p;
    Xoshiro rng(splitmix64(sd));
    int64_t lo = 0, hi = ncams - 1, kk;
    if (covis == 0) {
      kk = kmin + rng.below(kmax - kmin + 1);
    } else {
      const int64_t c = rng.below(ncams);
      lo = std::max<int64_t>(0, c - window);
      hi = std::min<int64_t>(ncams - 1, c + window);
      const int64_t g = (int64_t)std::floor(std::log(rng.uniform_open()) / std::log(1.0 - geom_p));
      kk = std::min<int64_t>(std::min<int64_t>(2 + g, kcap), hi - lo + 1);
    }
    kk = std::min<int64_t>(kk, hi - lo + 1);
    std::vector<int64_t> pool(hi - lo + 1);
    for (int64_t i = 0; i < (int64_t)pool.size(); ++i) pool[i] = lo + i;
    for (int64_t i = 0; i < kk; ++i) std::swap(pool[i], pool[i + rng.below((int64_t)pool.size() - i)]);
    std::vector<int64_t> sel(pool.begin(), pool.begin() + kk);
    std::sort(sel.begin(), sel.end());
    cams[p] = sel;
    k[p] = kk;
  }
  S->obs_ptr.assign(npoints + 1, 0);
  for (int64_t p = 0; p < npoints; ++p) S->obs_ptr[p + 1] = S->obs_ptr[p] + k[p];
  const int64_t nobs = S->obs_ptr[npoints];
  S->nobs = nobs;
  S->obs_cam.resize(nobs);
  S->Jc.resize(nobs * 12);
  S->Jp.resize(nobs * 6);
  S->r.resize(nobs * 2);
#pragma omp parallel for schedule(static, 1024)
  for (int64_t p = 0; p < npoints; ++p) {
    uint64_t sd = (seed ^ 0xD1B54A32D192ED03ull) * 0x9E3779B97F4A7C15ull + (uint64_t)p;
    Xoshiro rng(splitmix64(sd));
    const int64_t o0 = S->obs_ptr[p], kk = k[p], m = 2 * kk;
    // stacked point Jacobian, m x 3 column-major
    std::vector<double> A(m * 3);
    for (auto& x : A) x = rng.normal();
    if (sv_lo > 0) {
      double V[9];
      for (auto& x : V) x = rng.normal();
      orthonormalize(A.data(), (int)m, 3);
      orthonormalize(V, 3, 3);
      double sig[3];
      for (auto& x : sig) x = rng.loguniform(sv_lo, sv_hi);
      std::vector<double> B(m * 3, 0.0);   // Q diag(sig) V'
      for (int j = 0; j < 3; ++j)
        for (int t = 0; t < 3; ++t)
          for (int64_t i = 0; i < m; ++i) B[i + m * j] += A[i + m * t] * sig[t] * V[j + 3 * t];
      A.swap(B);
    }
    for (int64_t o = 0; o < kk; ++o) {
      const int64_t ob = o0 + o, cam = cams[p][o];
      S->obs_cam[ob] = cam;
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 2; ++i) S->Jp[ob * 6 + i + 2 * j] = A[(2 * o + i) + m * j];
      for (int j = 0; j < 6; ++j)
        for (int i = 0; i < 2; ++i) {
          double v = rng.normal();
          if (!cscale.empty()) v *= cscale[cam * 6 + j];
          S->Jc[ob * 12 + i + 2 * j] = v;
        }
      S->r[ob * 2 + 0] = rng.normal();
      S->r[ob * 2 + 1] = rng.normal();
    }
  }
  *out = S;
  return 0;
}

void bls_scene_destroy(bls_scene* S) { delete S; }

// Sizes: 0 ncams, 1 npoints, 2 nobs
int64_t bls_scene_size(const bls_scene* S, int what) {
  return what == 0 ? S->ncams : what == 1 ? S->npoints : S->nobs;
}

// Copy out: obs_ptr[npoints+1], obs_cam[nobs], Jc[nobs*12], Jp[nobs*6], r[nobs*2] (any may be NULL)
void bls_scene_arrays(const bls_scene* S, int64_t* obs_ptr, int64_t* obs_cam, double* Jc, double* Jp, double* r) {
  if (obs_ptr) std::memcpy(obs_ptr, S->obs_ptr.data(), S->obs_ptr.size() * 8);
  if (obs_cam) std::memcpy(obs_cam, S->obs_cam.data(), S->obs_cam.size() * 8);
  if (Jc) std::memcpy(Jc, S->Jc.data(), S->Jc.size() * 8);
  if (Jp) std::memcpy(Jp, S->Jp.data(), S->Jp.size() * 8);
  if (r) std::memcpy(r, S->r.data(), S->r.size() * 8);
}

// The elimination description in the caller's numbering: column blocks 0..ncams-1 are the cameras (size 6), then
// the points (size 3); one row block [camera, point] per observation, points in order. rb_ptr[nobs+1], rb_idx[2*nobs].
void bls_scene_description(const bls_scene* S, int64_t* blocksizes, uint8_t* eliminated, int64_t* rb_ptr, int64_t* rb_idx) {
  for (int64_t c = 0; c < S->ncams; ++c) { blocksizes[c] = 6; eliminated[c] = 0; }
  for (int64_t p = 0; p < S->npoints; ++p) { blocksizes[S->ncams + p] = 3; eliminated[S->ncams + p] = 1; }
  rb_ptr[0] = 0;
  for (int64_t p = 0; p < S->npoints; ++p)
    for (int64_t o = S->obs_ptr[p]; o < S->obs_ptr[p + 1]; ++o) {
      rb_idx[2 * o] = S->obs_cam[o];
      rb_idx[2 * o + 1] = S->ncams + p;
      rb_ptr[o + 1] = 2 * (o + 1);
    }
}

// Assemble H = J'J and b = J'r into the layout of a structure built from bls_scene_description:
//   position[nblocks]            layout position of each caller block (inverse of the structure's order)
//   eliminated_ptr, entry_retained, coffsets, eoffsets, boffsets_r, boffsets_e: the structure (0-based)
//   R: dense (R_dense_nr > 0: column-major nr x nr, both triangles of each diagonal block) or block-sparse on the
//      pattern (R_diag_start[r] = start of retained block r's diagonal block in the R data, d_r x d_r column-major)
// All outputs are zeroed first. Points are independent, so E, C and b_e are filled in parallel; R and b_r serially.
void bls_scene_assemble(const bls_scene* S, const int64_t* position, const int64_t* eliminated_ptr, const int64_t* entry_retained,
                        const int64_t* coffsets, const int64_t* eoffsets, const int64_t* boffsets_r, const int64_t* boffsets_e,
                        int64_t R_dense_nr, const int64_t* R_diag_start, double* E, int64_t E_len, double* C, int64_t C_len, double* R,
                        int64_t R_len, double* b_r, int64_t nr, double* b_e, int64_t ne) {
  std::memset(E, 0, E_len * 8);
  std::memset(C, 0, C_len * 8);
  std::memset(R, 0, R_len * 8);
  std::memset(b_r, 0, nr * 8);
  std::memset(b_e, 0, ne * 8);
  const int64_t nrb = S->ncams;
#pragma omp parallel for schedule(static, 1024)
  for (int64_t p = 0; p < S->npoints; ++p) {
    const int64_t e = position[S->ncams + p] - nrb;
    const int64_t eo = eoffsets[e], so = boffsets_e[e];
    for (int64_t o = S->obs_ptr[p]; o < S->obs_ptr[p + 1]; ++o) {
      const double* Jp = S->Jp.data() + o * 6;
      const double* Jc = S->Jc.data() + o * 12;
      const double* rr = S->r.data() + o * 2;
      const int64_t cam = position[S->obs_cam[o]];
      const int64_t* lo = entry_retained + eliminated_ptr[e];
      const int64_t* hi = entry_retained + eliminated_ptr[e + 1];
      const int64_t c = std::lower_bound(lo, hi, cam) - entry_retained;
      const int64_t co = coffsets[c];
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) E[eo + i + 3 * j] += Jp[2 * i] * Jp[2 * j] + Jp[2 * i + 1] * Jp[2 * j + 1];
      for (int j = 0; j < 6; ++j)
        for (int i = 0; i < 3; ++i) C[co + j * 3 + i] += Jp[2 * i] * Jc[2 * j] + Jp[2 * i + 1] * Jc[2 * j + 1];
      for (int i = 0; i < 3; ++i) b_e[so + i] += Jp[2 * i] * rr[0] + Jp[2 * i + 1] * rr[1];
    }
  }
  for (int64_t p = 0; p < S->npoints; ++p)
    for (int64_t o = S->obs_ptr[p]; o < S->obs_ptr[p + 1]; ++o) {
      const double* Jc = S->Jc.data() + o * 12;
      const double* rr = S->r.data() + o * 2;
      const int64_t cam = position[S->obs_cam[o]];
      const int64_t ro = boffsets_r[cam];
      for (int j = 0; j < 6; ++j)
        for (int i = 0; i < 6; ++i) {
          const double v = Jc[2 * i] * Jc[2 * j] + Jc[2 * i + 1] * Jc[2 * j + 1];
          if (R_dense_nr > 0) R[(ro + i) + (ro + j) * R_dense_nr] += v;
          else R[R_diag_start[cam] + i + 6 * j] += v;
        }
      for (int i = 0; i < 6; ++i) b_r[ro + i] += Jc[2 * i] * rr[0] + Jc[2 * i + 1] * rr[1];
    }
}

// Fill the raw Jacobian tables of a QR structure built from bls_scene_description with rowblocksizes 2 (the
// reference's block!/residual_block! writes, src/schur_jacobian.jl:368-387): observation o is row block o, its two rows
// at row_first[o] of table row_table[o]; its camera Jacobian goes to the columns of the camera's entry, its point
// Jacobian to the table's last three columns, its residual to the table's residual rows. Damping rows stay zero.
// position: layout position of each caller block; the cameras are the retained blocks.
int bls_scene_assemble_qr(const bls_scene* S, const int64_t* position, const int64_t* row_table, const int64_t* row_first,
                          const int64_t* table_ptr, const int64_t* entry_retained, const int64_t* entry_col, const int64_t* table_nrows,
                          const int64_t* table_ncols, const int64_t* raw_offsets, const int64_t* residual_offsets, double* Rw, int64_t Rw_len,
                          double* Rr, int64_t Rr_len) {
  std::memset(Rw, 0, Rw_len * 8);
  std::memset(Rr, 0, Rr_len * 8);
  int bad = 0;
#pragma omp parallel for schedule(static, 1024) reduction(| : bad)
  for (int64_t p = 0; p < S->npoints; ++p)
    for (int64_t o = S->obs_ptr[p]; o < S->obs_ptr[p + 1]; ++o) {
      const int64_t t = row_table[o], M = table_nrows[t], C = table_ncols[t] - 1, r0 = row_first[o];
      const int64_t cam = position[S->obs_cam[o]];
      const int64_t* lo = entry_retained + table_ptr[t];
      const int64_t* hi = entry_retained + table_ptr[t + 1];
      const int64_t* f = std::lower_bound(lo, hi, cam);
      if (f == hi || *f != cam || r0 + 2 > M || raw_offsets[t + 1] > Rw_len || residual_offsets[t + 1] > Rr_len) { bad = 1; continue; }
      const int64_t col = entry_col[f - entry_retained];
      double* T = Rw + raw_offsets[t];
      const double* Jc = S->Jc.data() + o * 12;
      const double* Jp = S->Jp.data() + o * 6;
      for (int j = 0; j < 6; ++j)
        for (int i = 0; i < 2; ++i) T[(col + j) * M + r0 + i] = Jc[2 * j + i];
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 2; ++i) T[(C - 3 + j) * M + r0 + i] = Jp[2 * j + i];
      for (int i = 0; i < 2; ++i) Rr[residual_offsets[t] + r0 + i] = S->r[o * 2 + i];
    }
  return bad ? -1 : 0;
}

}  // extern "C"
