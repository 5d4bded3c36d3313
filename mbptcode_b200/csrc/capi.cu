// C entry points of libmbpt_b200: orchestration of the route on the caller's
// stream over the caller's workspace. FP64 mode runs the N^3 products through
// cuBLAS DGEMM (the plain GPU path); mixed mode through the tcgen05 split
// engine (umma_gemm.cuh). The Cholesky factorisations use cuSOLVER in FP64.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <algorithm>
#include <tuple>
#include <vector>

#include "internal.h"

namespace mbpt {
int launch_pade_qp(const double *sigma, const double *pade_freq, int npade,
                   const double *eps_anchor, const double *xc, const int64_t *states,
                   int nstates, int64_t nocc, double mu, int greedy, const double *warm,
                   double *roots, double *z, int *flags, int *evals, cudaStream_t st);
int launch_pade_eval(const double *sigma, const double *pade_freq, int npade,
                     const int64_t *states, int nstates, int64_t nocc, double mu, int greedy,
                     const double *query, int nq, double *out, cudaStream_t st);
void launch_chi0_bar_seed(double *a, int64_t n, int nfreq, const double *scale,
                          cudaStream_t st);
void launch_sym_half(const double *in, double *out, int64_t n, cudaStream_t st);
void launch_xbar_update(const double *GoX, const double *GvX, const double *X, int64_t M,
                        int64_t n, int64_t nocc, const double *eps, double mu, double tau,
                        double *X_bar, double *eps_bar, cudaStream_t st);
void launch_mirror_lower_to_upper(double *a, int64_t n, cudaStream_t st);
void launch_lu_logdet(const double *LU, const int *piv, int64_t n, double *logdet, int *sign,
                      cudaStream_t st);
void launch_identity(double *a, int64_t n, cudaStream_t st);
void launch_minus_identity(double *a, int64_t n, cudaStream_t st);
void launch_diag(double *a, int64_t n, int nmat, double *diag, bool save, cudaStream_t st);
void launch_lower_copy(const double *A, int64_t lda, double *T, int ib, cudaStream_t st);
void launch_zero_strict_upper_cm(double *a, int64_t n, cudaStream_t st);
int launch_trtri_diag_blocks(double *A, int64_t n, int64_t lda, int nb, cudaStream_t st,
                             float *c_hi = nullptr, float *c_lo = nullptr, float *r_hi = nullptr,
                             float *r_lo = nullptr, int64_t ldp = 0);
void launch_strided_to_tf32(const double *src, int64_t rows, int64_t k, int64_t rs, int64_t cs,
                            float *hi, float *lo, int64_t rows_p, int64_t k_p, cudaStream_t st);
void launch_row_scaled_copy(const double *X, int64_t M, int64_t n, int64_t p, double *out,
                            cudaStream_t st);
void launch_linv_blocks_to_pairs(const double *Linv, int64_t step_stride, int64_t n,
                                 float *c_hi, float *c_lo, float *r_hi, float *r_lo,
                                 int64_t ldp, cudaStream_t st);
void launch_rowdot_f32(const float *R, int64_t ld_r, const double *X, int64_t ld_x, int64_t M,
                       int64_t S, double *out, cudaStream_t st);
void launch_col_scale(const double *Y, const double *v, int64_t nr, int64_t nc, double factor,
                      double *out, bool accumulate, cudaStream_t st);
void launch_cols_scaled_copy(const double *C, int64_t ldc, int64_t j0, const double *f,
                             double s, int64_t nr, int64_t nc, double *out, cudaStream_t st);
void launch_row_scale_acc(const double *a, int64_t lda, int64_t p, const double *b, int64_t nr,
                          int64_t nc, double *out, cudaStream_t st);
void launch_row_dot_into_col(const double *G, const double *X, int64_t nr, int64_t nc,
                             double *out, int64_t ldo, int64_t p, cudaStream_t st);
void launch_chol_copy_panel(const double *A, int64_t n, int64_t j0, int64_t m, int nbj,
                            int nmat, bool one_minus, double *P, cudaStream_t st);
int launch_chol_diag_block(const double *P, int64_t m, int nbj, double *A, int64_t n,
                           int64_t j0, int nmat, double *Linv, int *info, cudaStream_t st);
void launch_sigma_back_gather(const double *X, int64_t M, int64_t n, const int64_t *states,
                              int64_t S, const double *sl, const double *sg, double *Xs,
                              double *Xl, double *Xg, cudaStream_t st);
void launch_sigma_back_hadamard(double *go, double *gv, double *zt, double *al, double *ag,
                                int64_t total, cudaStream_t st);
void launch_scatter_cols(const double *T, int64_t M, int64_t S, const int64_t *states,
                         double scale, double *X_bar, int64_t n, cudaStream_t st);

namespace {
std::atomic<long long> g_launches{0};
}  // namespace

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {

constexpr int kAbiVersion = 2;

struct Handles {
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
};

Handles &handles(cudaStream_t st) {
  thread_local Handles h;
  if (!h.blas) {
    cublasCreate(&h.blas);
    cusolverDnCreate(&h.solver);
  }
  cublasSetStream(h.blas, st);
  cusolverDnSetStream(h.solver, st);
  return h;
}

// row-major C (m x n) = alpha op(A) op(B) + beta C
bool dgemm_rm(cublasHandle_t h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
              double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
              double beta, double *C, int64_t ldc) {
  return cublasDgemm(h, tb ? CUBLAS_OP_T : CUBLAS_OP_N, ta ? CUBLAS_OP_T : CUBLAS_OP_N,
                     static_cast<int>(n), static_cast<int>(m), static_cast<int>(k), &alpha, B,
                     static_cast<int>(ldb), A, static_cast<int>(lda), &beta, C,
                     static_cast<int>(ldc)) == CUBLAS_STATUS_SUCCESS;
}

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// The FP64 products of the reverse sweeps and of the rows beside the route
// (the adjoints, the AO self-energy, the contour's FP64 pieces) run on the
// int8 tensor cores by the Ozaki scheme (8 digits: FP64 level) unless
// MBPT_FP64_GEMM=cublas, which keeps cuBLAS DGEMMs. The forward sweeps' plain
// FP64 mode keeps native FP64 products; MBPT_MODE_FP64_INT8 puts them on the
// Ozaki product too. Read at every call.
bool ozaki_fp64_enabled() {
  const char *e = std::getenv("MBPT_FP64_GEMM");
  return !(e && std::strcmp(e, "cublas") == 0);
}

inline bool valid_mode(int m) {
  return m == MBPT_MODE_FP64 || m == MBPT_MODE_MIXED || m == MBPT_MODE_FP64_INT8;
}
// FP64-accurate modes: native FP64 products or the Ozaki emulation of them
inline bool fp64_mode(int m) { return m != MBPT_MODE_MIXED; }

// Grow-only scratch of the Ozaki GEMM, one per (device, stream): concurrent
// streams never share one. Growing waits for the stream's earlier work.
void *ozaki_scratch(cudaStream_t st, size_t bytes) {
  static std::mutex mu;
  static std::vector<std::tuple<int, cudaStream_t, void *, size_t>> held;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  for (auto &t : held) {
    if (std::get<0>(t) == dev && std::get<1>(t) == st) {
      if (std::get<3>(t) >= bytes) return std::get<2>(t);
      if (cudaStreamSynchronize(st) != cudaSuccess) return nullptr;
      cudaFree(std::get<2>(t));
      void *p = nullptr;
      if (cudaMalloc(&p, bytes) != cudaSuccess) {
        std::get<2>(t) = nullptr;
        std::get<3>(t) = 0;
        return nullptr;
      }
      std::get<2>(t) = p;
      std::get<3>(t) = bytes;
      return p;
    }
  }
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  held.emplace_back(dev, st, p, bytes);
  return p;
}

bool gemm_ozaki(cublasHandle_t h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
                double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
                double beta, double *C, int64_t ldc, const OzakiEpi *epi = nullptr) {
  cudaStream_t st = nullptr;
  if (cublasGetStream(h, &st) != CUBLAS_STATUS_SUCCESS) return false;
  const size_t bytes = ozaki_gemm_scratch_bytes(m, n, k, 8);
  void *ws = ozaki_scratch(st, bytes);
  if (!ws) return false;
  return ozaki_dgemm(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 8, ws, bytes,
                     nullptr, st, epi) == MBPT_OK;
}

bool gemm_f64(cublasHandle_t h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
              double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
              double beta, double *C, int64_t ldc) {
  if (!ozaki_fp64_enabled())
    return dgemm_rm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  return gemm_ozaki(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

// the forward sweeps' FP64 products: native in MBPT_MODE_FP64, on the Ozaki
// product in MBPT_MODE_FP64_INT8; `sym`: the n x n product is symmetric, and
// the Ozaki product forms its upper tiles only (the native one forms all)
bool gemm_mode(int mode, cublasHandle_t h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
               double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
               double beta, double *C, int64_t ldc, bool sym = false) {
  if (mode == MBPT_MODE_FP64_INT8) {
    OzakiEpi e;
    e.sym = sym;
    return gemm_ozaki(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, &e);
  }
  return dgemm_rm(h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

double *copy_weights(Arena &ar, const double *host, size_t count, cudaStream_t st) {
  double *d = ar.take<double>(count);
  if (d && host) cudaMemcpyAsync(d, host, count * sizeof(double), cudaMemcpyHostToDevice, st);
  return d;
}

struct Dims {
  int64_t M, n, nocc, nv, naux, Mp, Ap, Ko, Kv;
  Dims(int64_t M_, int64_t n_, int64_t nocc_, int64_t naux_)
      : M(M_), n(n_), nocc(nocc_), nv(n_ - nocc_), naux(naux_) {
    Mp = round_up(M, 128);
    Ap = round_up(naux, 128);
    Ko = round_up(nocc, 64);
    Kv = round_up(nv, 64);
  }
  bool ok() const { return M > 0 && n > nocc && nocc > 0 && naux > 0; }
};

// ---------------------------------------------------------------- chi0 sweep
struct Chi0Bufs {
  double *w;  // cosft_wt on the device
  // fp64
  double *Xo_s, *Xv_s, *Go, *Gv, *Y, *proj;
  // mixed
  bf16 *Dt_hi, *Dt_lo, *Pi_hi, *Pi_lo, *Z_hi, *Z_lo;
  float *Yo_hi, *Yo_lo, *Yv_hi, *Yv_lo;  // TF32 pairs of the G products
  float *proj32;
  double *eye;  // ntau x ntau identity for the optional proj copy
};

Chi0Bufs carve_chi0(Arena &ar, const Dims &d, int ntau, int nfreq, int mode, bool own_proj) {
  Chi0Bufs b{};
  b.w = ar.take<double>(static_cast<size_t>(nfreq) * ntau);
  if (fp64_mode(mode)) {
    b.Xo_s = ar.take<double>(d.M * d.nocc);
    b.Xv_s = ar.take<double>(d.M * d.nv);
    b.Go = ar.take<double>(d.M * d.M);
    b.Gv = ar.take<double>(d.M * d.M);
    b.Y = ar.take<double>(d.M * d.naux);
    if (own_proj) b.proj = ar.take<double>(static_cast<size_t>(ntau) * d.naux * d.naux);
  } else {
    b.Dt_hi = ar.take<bf16>(d.Ap * d.Mp);
    b.Dt_lo = ar.take<bf16>(d.Ap * d.Mp);
    b.Yo_hi = ar.take<float>(d.Mp * d.Ko);
    b.Yo_lo = ar.take<float>(d.Mp * d.Ko);
    b.Yv_hi = ar.take<float>(d.Mp * d.Kv);
    b.Yv_lo = ar.take<float>(d.Mp * d.Kv);
    b.Pi_hi = ar.take<bf16>(d.Mp * d.Mp);
    b.Pi_lo = ar.take<bf16>(d.Mp * d.Mp);
    b.Z_hi = ar.take<bf16>(d.Ap * d.Mp);
    b.Z_lo = ar.take<bf16>(d.Ap * d.Mp);
    b.proj32 = ar.take<float>(static_cast<size_t>(ntau) * d.Ap * d.Ap);
    b.eye = ar.take<double>(static_cast<size_t>(ntau) * ntau);
  }
  return b;
}

int chi0_run(const double *X, const Dims &d, const double *eps, double mu, const double *D,
             const double *tau, int ntau, const double *cw, int nfreq, int mode, double *chi0,
             double *proj_out, Arena &ar, int *err, cudaStream_t st) {
  Chi0Bufs b = carve_chi0(ar, d, ntau, nfreq, mode, proj_out == nullptr);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cudaMemcpyAsync(b.w, cw, sizeof(double) * nfreq * ntau, cudaMemcpyHostToDevice, st);
  const int64_t a2 = d.naux * d.naux;
  if (fp64_mode(mode)) {
    double *proj = proj_out ? proj_out : b.proj;
    cublasHandle_t h = handles(st).blas;
    for (int k = 0; k < ntau; ++k) {
      launch_scaled_branches(X, d.M, d.n, d.nocc, eps, mu, tau[k], 1.0, b.Xo_s, b.Xv_s, st);
      // G_occ = (X_o e^{e_o tau}) X_o^T, G_virt likewise (MBPTcode space_time.py:525-526)
      if (!gemm_mode(mode, h, false, true, d.M, d.M, d.nocc, 1.0, b.Xo_s, d.nocc, X, d.n, 0.0,
                     b.Go, d.M) ||
          !gemm_mode(mode, h, false, true, d.M, d.M, d.nv, 1.0, b.Xv_s, d.nv, X + d.nocc, d.n,
                     0.0, b.Gv, d.M))
        return MBPT_ERR_CUDA;
      launch_hadamard(b.Go, b.Gv, d.M * d.M, st);
      if (!gemm_mode(mode, h, false, false, d.M, d.naux, d.M, 1.0, b.Go, d.M, D, d.naux, 0.0,
                     b.Y, d.naux) ||
          !gemm_mode(mode, h, true, false, d.naux, d.naux, d.M, -2.0, D, d.naux, b.Y, d.naux,
                     0.0, proj + k * a2, d.naux, true))
        return MBPT_ERR_CUDA;
    }
    launch_transform<double>(proj, a2, d.naux, d.naux, d.naux, b.w, nfreq, ntau, chi0, a2,
                             d.naux, st);
  } else {
    launch_split_pad<double>(D, d.M, d.naux, d.naux, 1.f, b.Dt_hi, b.Dt_lo, d.Mp, d.Mp, d.Ap,
                             true, st);
    // G_occ and G_virt in TF32x3: their K sums cancel (off-diagonal entries
    // are ~sqrt(K) below the summed terms), which the BF16 split would carry
    // into chi0 at ~1e-4 relative; the D^T Pi D products stay BF16x3
    SplitMat Yo{b.Yo_hi, b.Yo_lo, d.Mp, d.Ko, d.Ko, true};
    SplitMat Yv{b.Yv_hi, b.Yv_lo, d.Mp, d.Kv, d.Kv, true};
    SplitMat Dt{b.Dt_hi, b.Dt_lo, d.Ap, d.Mp, d.Mp};
    SplitMat Pi{b.Pi_hi, b.Pi_lo, d.Mp, d.Mp, d.Mp};
    SplitMat Z{b.Z_hi, b.Z_lo, d.Ap, d.Mp, d.Mp};
    for (int k = 0; k < ntau; ++k) {
      launch_prep_branches_tf32(X, d.M, d.n, d.nocc, eps, mu, tau[k], b.Yo_hi, b.Yo_lo, d.Ko,
                                b.Yv_hi, b.Yv_lo, d.Kv, d.Mp, st);
      umma::EpiArgs e;
      // Pi = (Y_o Y_o^T) o (Y_v Y_v^T), split for the next product
      e.out0_hi = b.Pi_hi;
      e.out0_lo = b.Pi_lo;
      e.ld_out = d.Mp;
      SplitMat A2[2] = {Yo, Yv};
      // Pi is symmetric: the tiles on and above the diagonal, mirrored by the epilogue
      int rc = gemm_split(umma::EPI_HADAMARD_SPLIT, 2, A2, A2, d.Mp, d.Mp, e, err, st,
                          umma::BAND_UPPER);
      if (rc) return rc;
      // Z = D^T Pi  (= (Pi D)^T, Pi symmetric)
      e = umma::EpiArgs();
      e.out0_hi = b.Z_hi;
      e.out0_lo = b.Z_lo;
      e.ld_out = d.Mp;
      rc = gemm_split(umma::EPI_SPLIT, 1, &Dt, &Pi, d.Ap, d.Mp, e, err, st);
      if (rc) return rc;
      // proj = -2 D^T Z^T
      e = umma::EpiArgs();
      e.outf = b.proj32 + k * d.Ap * d.Ap;
      e.ld_outf = d.Ap;
      e.alpha = -2.f;
      // proj = -2 D^T Pi D is symmetric: upper tiles, mirrored
      rc = gemm_split(umma::EPI_F32, 1, &Dt, &Z, d.Ap, d.Ap, e, err, st, umma::BAND_UPPER);
      if (rc) return rc;
    }
    launch_transform<float>(b.proj32, d.Ap * d.Ap, d.Ap, d.naux, d.naux, b.w, nfreq, ntau,
                            chi0, a2, d.naux, st);
    if (proj_out) {
      std::vector<double> eye(static_cast<size_t>(ntau) * ntau, 0.0);
      for (int k = 0; k < ntau; ++k) eye[k * ntau + k] = 1.0;
      cudaMemcpyAsync(b.eye, eye.data(), sizeof(double) * eye.size(), cudaMemcpyHostToDevice,
                      st);
      launch_transform<float>(b.proj32, d.Ap * d.Ap, d.Ap, d.naux, d.naux, b.eye, ntau, ntau,
                              proj_out, a2, d.naux, st);
    }
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// --------------------------------------------------------------------- Dyson
// Block size of the LAUUM below; its DGEMM/DSYRK updates carry the flops.
constexpr int64_t kLauumBlock = 512;

// Diagonal blocks of the triangular inverse, inverted all at once in shared
// memory (one CTA per block); the recursion above them turns the rest into
// dense products.
constexpr int64_t kTrtriLeaf = 128;

// Mixed-mode scratch of the inverse: TF32 hi/lo pair arrays, np x np each
// (np = n rounded up to 128), zero outside what the recursion writes.
//   LR: rows of the factor L (row i along k);
//   IC: columns of L^-1 as rows, IC(j, k) = L^-1(k, j);
//   IR: rows of L^-1, IR(i, k) = L^-1(i, k);
//   TT: one product's T^T between the two products of a recursion node.
struct PairScratch {
  float *lr_hi = nullptr, *lr_lo = nullptr, *ic_hi = nullptr, *ic_lo = nullptr;
  float *ir_hi = nullptr, *ir_lo = nullptr, *tt_hi = nullptr, *tt_lo = nullptr;
  int64_t np = 0;
};

// In place: the lower-triangular column-major block at A (n x n, leading
// dimension lda, zeros above its diagonal, its kTrtriLeaf diagonal blocks
// already inverted) becomes its inverse, by
// [[L11, 0], [L21, L22]]^-1 = [[L11^-1, 0], [-L22^-1 L21 L11^-1, L22^-1]]
// with both halves inverted first (n1 a multiple of kTrtriLeaf keeps the
// leaves on the diagonal blocks). T holds (n - n1) x n1 doubles. FP64 DGEMMs.
int trtri_rec(Handles &h, double *A, int64_t n, int64_t lda, double *T) {
  if (n <= kTrtriLeaf) return MBPT_OK;
  const int64_t n1 = round_up(n / 2, kTrtriLeaf), n2 = n - n1;
  double *L11 = A, *L21 = A + n1, *L22 = A + n1 + n1 * lda;
  int rc = trtri_rec(h, L11, n1, lda, T);
  if (rc) return rc;
  rc = trtri_rec(h, L22, n2, lda, T);
  if (rc) return rc;
  const double one = 1.0, zero = 0.0, minus = -1.0;
  const int i1 = static_cast<int>(n1), i2 = static_cast<int>(n2), il = static_cast<int>(lda);
  // T = L21 L11^-1, then L21 <- -L22^-1 T
  if (cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, i2, i1, i1, &one, L21, il, L11, il, &zero,
                  T, i2) != CUBLAS_STATUS_SUCCESS ||
      cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, i2, i1, i2, &minus, L22, il, T, i2, &zero,
                  L21, il) != CUBLAS_STATUS_SUCCESS)
    return MBPT_ERR_CUDA;
  return MBPT_OK;
}

// The same recursion on TF32 pairs over the whole n x n factor (diagonal
// kTrtriLeaf blocks already in IC/IR, the factor's rows in LR), level by
// level: the nodes of one depth are independent, so each depth is two grouped
// launches, deepest first. Each node's products have epilogues that write
// pairs straight into the layouts the next products read, so nothing is
// converted between them. With the engine forming P = A_e B_e^T row by row of
// A_e, for the node [o, o + n) split at n1:
//   P1 = T^T = (L11^-1)^T L21^T:  A_e = IC rows (zero for k < row: K from m0),
//        B_e = LR rows of L21; stored as pairs in TT rows [o, o + n1);
//   P2 = L21'^T = -(T^T) (L22^-1)^T: A_e = TT, B_e = IR rows of L22^-1 (zero
//        for k > row: K up to the tile's end); stored into IC and, transposed,
//        into IR.
// Nodes of one depth cover disjoint rows, so their TT blocks do not overlap.
void collect_nodes(int64_t o, int64_t n, size_t depth,
                   std::vector<std::vector<std::pair<int64_t, int64_t>>> &levels) {
  if (n <= kTrtriLeaf) return;
  if (levels.size() <= depth) levels.resize(depth + 1);
  levels[depth].push_back({o, n});
  const int64_t n1 = round_up(n / 2, kTrtriLeaf);
  collect_nodes(o, n1, depth + 1, levels);
  collect_nodes(o + n1, n - n1, depth + 1, levels);
}

int trtri_pairs(const PairScratch &s, int64_t n, int *err, cudaStream_t st) {
  std::vector<std::vector<std::pair<int64_t, int64_t>>> levels;
  collect_nodes(0, n, 0, levels);
  const int64_t ld = s.np;
  const SplitMat IC{s.ic_hi, s.ic_lo, ld, ld, ld, true}, IR{s.ir_hi, s.ir_lo, ld, ld, ld, true};
  const SplitMat LR{s.lr_hi, s.lr_lo, ld, ld, ld, true}, TT{s.tt_hi, s.tt_lo, ld, ld, ld, true};
  std::vector<GemmGroup> g1, g2;
  for (size_t d = levels.size(); d-- > 0;) {
    g1.clear();
    g2.clear();
    for (const auto &node : levels[d]) {
      const int64_t o = node.first, nn = node.second;
      const int64_t n1 = round_up(nn / 2, kTrtriLeaf), n2 = nn - n1, n2p = round_up(n2, 128);
      g1.push_back({n1, n2p, n1, o, o, o + n1, o, o * ld, 0});
      g2.push_back({n1, n2p, n2, o, 0, o + n1, o + n1, o * ld + o + n1, (o + n1) * ld + o});
    }
    umma::EpiArgs e1;
    e1.p_hi = s.tt_hi;
    e1.p_lo = s.tt_lo;
    e1.ld_p = ld;
    e1.alpha = 1.f;
    int rc = gemm_split_grouped(umma::EPI_TF32_PAIR, IC, LR, g1.data(),
                                static_cast<int>(g1.size()), e1, err, st, umma::BAND_K_FROM_M);
    if (rc) return rc;
    umma::EpiArgs e2;
    e2.p_hi = s.ic_hi;
    e2.p_lo = s.ic_lo;
    e2.ld_p = ld;
    e2.t_hi = s.ir_hi;
    e2.t_lo = s.ir_lo;
    e2.ld_t = ld;
    e2.alpha = -1.f;
    rc = gemm_split_grouped(umma::EPI_TF32_PAIR, TT, IR, g2.data(), static_cast<int>(g2.size()),
                            e2, err, st, umma::BAND_K_TO_N);
    if (rc) return rc;
  }
  return MBPT_OK;
}

struct TimingTag {
  explicit TimingTag(int tag) { timing_tag(tag); }
  ~TimingTag() { timing_tag(-1); }
};

// W - I from the Cholesky factor L of 1 - chi0 (column-major lower, in place;
// the row-major upper triangle of the buffer). FP64 mode: the diagonal blocks
// of L^-1 in shared memory, the recursion above on DGEMMs, then (L^-1)^T L^-1
// by a blocked LAUUM on cuBLAS level 3 (LAPACK's blocking) into the same
// triangle, which the caller mirrors and shifts by -I; this replaces potri,
// whose LAUUM half runs far below DGEMM speed. Mixed mode (`pairs`): L^-1 as
// TF32 pairs by the tensor-core recursion, then W = (L^-1)^T L^-1 on the
// tensor cores over the tiles on and above the diagonal (rows of (L^-1)^T
// vanish for k < row), W - I written whole (returns with *full = true).
int spd_inverse_from_factor(Handles &h, double *L, int64_t n, double *T, double *Tr,
                            const PairScratch *pairs, int *err, bool *full, cudaStream_t st,
                            const double *diag_inv = nullptr, int64_t diag_inv_stride = 0) {
  *full = false;
  TimingTag tag(kTimingDyson);
  if (pairs) {
    const PairScratch &s = *pairs;
    const int64_t np = s.np, kp = round_up(n, 32);
    // rows of L (its upper triangle is never read)
    launch_strided_to_tf32(L, n, n, 1, n, s.lr_hi, s.lr_lo, np, np, st);
    int rc = MBPT_OK;
    if (diag_inv)
      // the batched factorisation kept its inverted 128 x 128 diagonal blocks
      launch_linv_blocks_to_pairs(diag_inv, diag_inv_stride, n, s.ic_hi, s.ic_lo, s.ir_hi,
                                  s.ir_lo, np, st);
    else
      rc = launch_trtri_diag_blocks(L, n, n, static_cast<int>(kTrtriLeaf), st, s.ic_hi,
                                    s.ic_lo, s.ir_hi, s.ir_lo, np);
    if (rc) return rc;
    rc = trtri_pairs(s, n, err, st);
    if (rc) return rc;
    // W - I straight into the factor's buffer as FP64 (row-major W(j, i) is
    // the column-major W(i, j) the caller expects; W is symmetric anyway),
    // tiles above the diagonal mirrored by the epilogue
    SplitMat Ae{s.ic_hi, s.ic_lo, np, kp, np, true};
    umma::EpiArgs e;
    e.outd = L;
    e.ld_outd = n;
    e.nd = static_cast<int>(n);
    e.shift = 1.0;
    e.alpha = 1.f;
    rc = gemm_split(umma::EPI_F64_SYM, 1, &Ae, &Ae, np, np, e, err, st,
                    umma::BAND_K_FROM_M | umma::BAND_K_FROM_N | umma::BAND_UPPER);
    if (rc) return rc;
    *full = true;
    return MBPT_OK;
  }
  // the dense products of the recursion need zeros above the diagonal
  launch_zero_strict_upper_cm(L, n, st);
  int rc = launch_trtri_diag_blocks(L, n, n, static_cast<int>(kTrtriLeaf), st);
  if (rc) return rc;
  rc = trtri_rec(h, L, n, n, Tr);
  if (rc) return rc;
  const double one = 1.0, zero = 0.0;
  const int lda = static_cast<int>(n);
  for (int64_t i = 0; i < n; i += kLauumBlock) {
    const int ib = static_cast<int>(std::min(kLauumBlock, n - i));
    const int ii = static_cast<int>(i);
    double *Aii = L + i + i * n;
    // A(i:i+ib, 0:i) = A(i:i+ib, i:i+ib)^T A(i:i+ib, 0:i)
    if (ii > 0 &&
        cublasDtrmm(h.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                    CUBLAS_DIAG_NON_UNIT, ib, ii, &one, Aii, lda, L + i, lda, L + i, lda) !=
            CUBLAS_STATUS_SUCCESS)
      return MBPT_ERR_CUDA;
    // A(i:i+ib, i:i+ib) = L11^T L11 from a copy with its strict upper part cleared
    launch_lower_copy(Aii, n, T, ib, st);
    if (cublasDsyrk(h.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, ib, ib, &one, T, ib, &zero,
                    Aii, lda) != CUBLAS_STATUS_SUCCESS)
      return MBPT_ERR_CUDA;
    if (i + ib < n) {
      const int rest = static_cast<int>(n - i - ib);
      double *Abelow = L + (i + ib) + i * n;  // A(i+ib:n, i:i+ib)
      if (ii > 0 && cublasDgemm(h.blas, CUBLAS_OP_T, CUBLAS_OP_N, ib, ii, rest, &one, Abelow,
                                lda, L + (i + ib), lda, &one, L + i, lda) !=
                        CUBLAS_STATUS_SUCCESS)
        return MBPT_ERR_CUDA;
      if (cublasDsyrk(h.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, ib, rest, &one, Abelow, lda,
                      &one, Aii, lda) != CUBLAS_STATUS_SUCCESS)
        return MBPT_ERR_CUDA;
    }
  }
  return MBPT_OK;
}

constexpr int kCholNb = 128;     // block columns of the batched Cholesky
constexpr int kBatchedCholMin = 4;  // frequencies from which the batch beats one potrf each

// Left-looking blocked Cholesky of nmat column-major n x n SPD matrices at
// once (A_f = L_f L_f^T, L_f in the lower triangle, the strict upper triangle
// untouched, info_f as potrf reports it). Per 128-column step j0, for all
// matrices in one launch each: the block column is copied to P, updated by
// one strided-batched DGEMM P -= L[j0:, :j0] L[j0:j0+nb, :j0]^T (inner
// dimension j0, so the FP64 GEMMs run long), its diagonal block factorised
// and inverted in shared memory, and the panel below it formed by a second
// batched DGEMM, L[j0+nb:, j0-block] = P_below L_jj^-T. Every launch carries
// the whole batch, so the latency-bound diagonal blocks cost one launch per
// step for all frequencies. P: nmat * n * kCholNb doubles; Linv: nmat *
// kCholNb^2 doubles per step, step j at Linv + j * linv_step_stride (0: every
// step in the same place); info: nmat ints, zeroed by the caller.
// one_minus: A holds chi0 and the factorised matrices are I - A_f, formed
// where each block column is first read (A's strict upper triangle keeps
// chi0, its diagonal and lower triangle become the factor).
// The Ozaki-scheme update's buffers for one batch (null planes: the updates
// run as cuBLAS DGEMMs): the int8 digit planes, 2^e_r per row, exact row norms.
struct OzakiChol {
  int8_t *planes = nullptr;
  double *scale = nullptr;
  double *rowsq = nullptr;   // running FP64 row norms, nmat x n
  int slices = 8;
  int *err = nullptr;
};

int chol_batched(double *A, int64_t n, int nmat, int *info, double *P, double *Linv,
                 cublasHandle_t h, cudaStream_t st, int64_t linv_step_stride = 0,
                 const OzakiChol *oz = nullptr, bool one_minus = false) {
  const long long n2 = static_cast<long long>(n) * n;
  const double one = 1.0, minus = -1.0, zero = 0.0;
  const bool ozaki = oz && oz->planes;
  if (ozaki) {
    int rc = ozaki_chol_scales(A, n, nmat, oz->scale, oz->rowsq, one_minus, st);
    if (rc) return rc;
  }
  for (int64_t j0 = 0; j0 < n; j0 += kCholNb) {
    const int nbj = static_cast<int>(std::min<int64_t>(kCholNb, n - j0));
    const int64_t m = n - j0;
    launch_chol_copy_panel(A, n, j0, m, nbj, nmat, one_minus, P, st);
    if (ozaki) {
      int rc = ozaki_chol_update(A, n, nmat, j0, nbj, P, oz->scale, oz->planes, oz->slices,
                                 oz->rowsq, oz->err, st);
      if (rc) return rc;
    } else if (j0 > 0 &&
               cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_T, static_cast<int>(m), nbj,
                                         static_cast<int>(j0), &minus, A + j0,
                                         static_cast<int>(n), n2, A + j0, static_cast<int>(n),
                                         n2, &one, P, static_cast<int>(m),
                                         static_cast<long long>(m) * nbj,
                                         nmat) != CUBLAS_STATUS_SUCCESS) {
      return MBPT_ERR_CUDA;
    }
    double *Lj = Linv + (j0 / kCholNb) * linv_step_stride;
    int rc = launch_chol_diag_block(P, m, nbj, A, n, j0, nmat, Lj, info, st);
    if (rc) return rc;
    const int64_t mb = m - nbj;
    if (mb > 0 &&
        cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_T, static_cast<int>(mb), nbj, nbj,
                                  &one, P + nbj, static_cast<int>(m),
                                  static_cast<long long>(m) * nbj, Lj, kCholNb,
                                  static_cast<long long>(kCholNb) * kCholNb, &zero,
                                  A + j0 * n + j0 + nbj, static_cast<int>(n), n2,
                                  nmat) != CUBLAS_STATUS_SUCCESS)
      return MBPT_ERR_CUDA;
    // the block column is final: cut it into digit planes for the later steps
    if (ozaki && j0 + nbj < n) {
      int rc2 = ozaki_chol_slice(A, n, nmat, j0, nbj, oz->scale, oz->planes, oz->slices,
                                 oz->rowsq, st);
      if (rc2) return rc2;
    }
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// The batched Cholesky's trailing updates: on the int8 tensor cores (the
// Ozaki scheme) in mixed mode, as native FP64 DGEMMs in FP64 mode (the plain
// FP64 path the mixed one is measured against). Digits per operand: in
// mixed mode 6 signed 8-bit digits (the log-determinant within 1e-14 of
// LAPACK, W from the factor within ~2e-12 of its largest entry; W is formed
// from it by TF32x3 products there), 8 when forced in FP64 mode
// (W within ~1e-14). MBPT_DYSON_OZAKI=1 / =0 forces the int8 path or the
// DGEMMs in both modes, MBPT_DYSON_OZAKI_SLICES=6 / 7 / 8 the digits (6:
// signed 8-bit digits, whose exact int32 level sums hold K below 22 016, so
// larger matrices take 7). Read at every call, so the size query and the call
// that follows it must see the same setting.
int ozaki_slices(int mode, int64_t n) {
  const char *e = std::getenv("MBPT_DYSON_OZAKI");
  const bool on = e ? std::atoi(e) != 0 : mode != MBPT_MODE_FP64;
  if (!on) return 0;
  const char *k = std::getenv("MBPT_DYSON_OZAKI_SLICES");
  int v = k ? std::atoi(k) : (mode == MBPT_MODE_MIXED ? 6 : 8);
  if (v == 6 && n > kOzakiEightBitMaxK) v = 7;
  return (v == 6 || v == 7 || v == 8) ? v : 8;
}

// Mixed mode: the tensor-core inverses of that many frequencies run at once,
// each on its own side stream with its own TF32 pair scratch (8 n_p^2 floats):
// the recursion's deep levels are small products that leave most of the GPU
// idle when one frequency runs alone. MBPT_DYSON_INVERSE_STREAMS (1 to 4,
// default 4), read once per process so that the size query and the call see
// the same count.
constexpr int kMaxInverseStreams = 4;
int inverse_streams() {
  static const int v = [] {
    const char *e = std::getenv("MBPT_DYSON_INVERSE_STREAMS");
    const int k = e ? std::atoi(e) : kMaxInverseStreams;
    return std::max(1, std::min(kMaxInverseStreams, k));
  }();
  return v;
}

bool batched_chol_enabled(int nfreq) {
  // MBPT_DYSON_BATCHED=0 keeps one cuSOLVER potrf per frequency
  static const int env = [] {
    const char *e = std::getenv("MBPT_DYSON_BATCHED");
    return e ? std::atoi(e) : 1;
  }();
  return env != 0 && nfreq >= kBatchedCholMin;
}

struct DysonBufs {
  int *info;
  int *piv;
  double *work;
  double *work2;  // the second factor stream's cuSOLVER workspace
  double *rhs;   // n x n right-hand side of the LU inverse of a failed frequency
  double *diag;  // nfreq x n diagonals of 1 - chi0, which the factorisation overwrites
  double *T;     // diagonal-block scratch of the LAUUM
  PairScratch pairs[kMaxInverseStreams];  // mixed mode: one per inverse stream
  int npairs = 0;
  double *chol_P = nullptr, *chol_Linv = nullptr;  // batched Cholesky scratch
  int8_t *oz_planes = nullptr;                       // Ozaki digit planes (all frequencies)
  double *oz_scale = nullptr, *oz_rowsq = nullptr;
  int oz_slices = 0;
  int lwork;
};

int dyson_lwork(int64_t n) {
  cudaStream_t st = nullptr;
  Handles &h = handles(st);
  int l1 = 0, l3 = 0;
  cusolverDnDpotrf_bufferSize(h.solver, CUBLAS_FILL_MODE_LOWER, static_cast<int>(n), nullptr,
                              static_cast<int>(n), &l1);
  cusolverDnDgetrf_bufferSize(h.solver, static_cast<int>(n), static_cast<int>(n), nullptr,
                              static_cast<int>(n), &l3);
  return l1 > l3 ? l1 : l3;
}

DysonBufs carve_dyson(Arena &ar, int64_t n, int nfreq, int mode = MBPT_MODE_FP64) {
  DysonBufs b{};
  b.lwork = dyson_lwork(n);
  b.info = ar.take<int>(nfreq + 1);
  b.piv = ar.take<int>(n);
  b.work = ar.take<double>(b.lwork > 0 ? b.lwork : 1);
  b.work2 = ar.take<double>(b.lwork > 0 ? b.lwork : 1);
  b.rhs = ar.take<double>(n * n);
  b.diag = ar.take<double>(n * static_cast<int64_t>(nfreq));
  b.T = ar.take<double>(kLauumBlock * kLauumBlock);
  if (batched_chol_enabled(nfreq)) {
    b.chol_P = ar.take<double>(static_cast<int64_t>(nfreq) * n * kCholNb);
    // every step's inverted diagonal blocks are kept: the mixed inverse reads them
    const int64_t steps = (n + kCholNb - 1) / kCholNb;
    b.chol_Linv = ar.take<double>(steps * nfreq * kCholNb * kCholNb);
    b.oz_slices = ozaki_slices(mode, n);
    if (b.oz_slices) {
      b.oz_planes = ar.take<int8_t>(ozaki_planes_bytes(n, nfreq, b.oz_slices));
      b.oz_scale = ar.take<double>(static_cast<int64_t>(nfreq) * n);
      b.oz_rowsq = ar.take<double>(static_cast<int64_t>(nfreq) * n);
    }
  }
  if (mode == MBPT_MODE_MIXED) {
    const int64_t np = round_up(n, 128), cap = np * np;
    b.npairs = std::min(inverse_streams(), std::max(1, nfreq));
    for (int i = 0; i < b.npairs; ++i) {
      PairScratch &q = b.pairs[i];
      q.np = np;
      for (float **f : {&q.lr_hi, &q.lr_lo, &q.ic_hi, &q.ic_lo, &q.ir_hi, &q.ir_lo, &q.tt_hi,
                        &q.tt_lo})
        *f = ar.take<float>(cap);
    }
  }
  return b;
}

// Per host thread and device: a side stream on which the inverse of one
// frequency runs while the next frequency factorises on the caller's stream,
// one event per frequency (its factor, log-determinant and info word are
// done) and a pinned host copy of the info words.
struct DysonPipe {
  cudaStream_t side = nullptr;
  cudaEvent_t join = nullptr;
  // the inverses' own cuBLAS handle (bound to `side`): the caller's handle
  // may still be running a later wave's factorisation on the caller's stream
  cublasHandle_t blas_side = nullptr;
  // mixed mode's further inverse streams (index i + 1 of the inverse streams)
  std::vector<cudaStream_t> isides;
  std::vector<cudaEvent_t> ijoin;
  // second factor stream: odd frequencies factorise there with their own
  // cuSOLVER handle, so that two Cholesky factorisations (latency-bound
  // panels between DGEMM-bound updates) share the GPU
  cudaStream_t fac2 = nullptr;
  cusolverDnHandle_t solver2 = nullptr;
  cublasHandle_t blas2 = nullptr;  // the second half of a batched factorisation
  cudaEvent_t fork = nullptr, join2 = nullptr;
  int nfac = 1;
  // groups of the batched factorisation (MBPT_DYSON_CHOL_GROUPS, default 4):
  // group 0 on the caller's stream, group 1 on fac2, the rest on these
  int groups = 2;
  std::vector<cudaStream_t> xs;
  std::vector<cublasHandle_t> xb;
  std::vector<cudaEvent_t> xj;
  std::vector<cudaEvent_t> ev;
  int *info = nullptr;  // pinned host, `cap` ints
  int cap = 0;
  bool ok = false;
};

DysonPipe *dyson_pipe(int nfreq) {
  thread_local std::vector<std::pair<int, DysonPipe>> pipes;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  DysonPipe *p = nullptr;
  for (auto &e : pipes)
    if (e.first == dev) p = &e.second;
  if (!p) {
    pipes.emplace_back(dev, DysonPipe{});
    p = &pipes.back().second;
    p->ok = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming) == cudaSuccess &&
            cublasCreate(&p->blas_side) == CUBLAS_STATUS_SUCCESS &&
            cublasSetStream(p->blas_side, p->side) == CUBLAS_STATUS_SUCCESS;
    // MBPT_DYSON_FACTOR_STREAMS=1 keeps every factorisation on the caller's stream
    const char *env = std::getenv("MBPT_DYSON_FACTOR_STREAMS");
    p->nfac = (env && std::atoi(env) == 1) ? 1 : 2;
    if (p->ok && p->nfac == 2)
      p->ok = cudaStreamCreateWithFlags(&p->fac2, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&p->join2, cudaEventDisableTiming) == cudaSuccess &&
              cusolverDnCreate(&p->solver2) == CUSOLVER_STATUS_SUCCESS &&
              cusolverDnSetStream(p->solver2, p->fac2) == CUSOLVER_STATUS_SUCCESS &&
              cublasCreate(&p->blas2) == CUBLAS_STATUS_SUCCESS &&
              cublasSetStream(p->blas2, p->fac2) == CUBLAS_STATUS_SUCCESS;
    for (int i = 1; p->ok && i < kMaxInverseStreams; ++i) {
      cudaStream_t s = nullptr;
      cudaEvent_t e = nullptr;
      p->ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
      p->isides.push_back(s);
      p->ijoin.push_back(e);
    }
    const char *genv = std::getenv("MBPT_DYSON_CHOL_GROUPS");
    const int g = genv ? std::atoi(genv) : 4;
    p->groups = p->nfac == 2 ? std::max(1, std::min(6, g)) : 1;
    for (int i = 2; p->ok && i < p->groups; ++i) {
      cudaStream_t xs = nullptr;
      cublasHandle_t xb = nullptr;
      cudaEvent_t xj = nullptr;
      p->ok = cudaStreamCreateWithFlags(&xs, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&xj, cudaEventDisableTiming) == cudaSuccess &&
              cublasCreate(&xb) == CUBLAS_STATUS_SUCCESS &&
              cublasSetStream(xb, xs) == CUBLAS_STATUS_SUCCESS;
      p->xs.push_back(xs);
      p->xb.push_back(xb);
      p->xj.push_back(xj);
    }
  }
  while (p->ok && static_cast<int>(p->ev.size()) < nfreq) {
    cudaEvent_t e = nullptr;
    p->ok = cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
    if (p->ok) p->ev.push_back(e);
  }
  if (p->ok && p->cap < nfreq) {
    if (p->info) cudaFreeHost(p->info);
    p->info = nullptr;
    p->ok = cudaHostAlloc(reinterpret_cast<void **>(&p->info), sizeof(int) * nfreq,
                          cudaHostAllocPortable) == cudaSuccess;
    p->cap = p->ok ? nfreq : 0;
  }
  return p->ok ? p : nullptr;
}

// Factorise the frequencies on two streams (even ones on `st`, odd ones on the
// pipe's second factor stream, two ahead of the host); as soon as frequency
// f's info word is on the host, its inverse goes to the side stream, so that
// the tensor-core (or DGEMM) inverse of f overlaps the FP64 Cholesky
// factorisations of f + 1 and f + 2. A frequency that is not positive definite
// falls back to LU with every stream drained first. The caller's stream waits
// for the other two at the end.
// info_dev_out null: the host reads each frequency's info word before its
// inverse (a positive definite frequency's W from the factor, any other by
// LU). Non-null: no host wait; every frequency's inverse is issued from its
// factor and the info words land in info_dev_out, where a nonzero word marks
// a frequency whose W - I and log-determinant are not valid.
int dyson_run(double *chi0, int64_t n, int nfreq, int want_w, double *logdet, double *trace,
              int *info_host, int *sign_host, Arena &ar, cudaStream_t st,
              int mode = MBPT_MODE_FP64, int *err = nullptr, int *info_dev_out = nullptr) {
  const bool deferred = info_dev_out != nullptr;
  DysonBufs b = carve_dyson(ar, n, nfreq, mode);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  Handles &h = handles(st);
  DysonPipe *pp = dyson_pipe(nfreq);
  if (!pp) return MBPT_ERR_CUDA;
  const int ni = static_cast<int>(n);
  // many frequencies: one batched factorisation of all of them, then the
  // per-frequency loop below only reads their info words
  const bool batched = b.chol_P != nullptr;
  // the batch forms 1 - chi0 where it first reads each block column (no pass
  // of its own over the matrices); one potrf per frequency needs it whole
  if (batched)
    launch_trace(chi0, n, nfreq, trace, st);
  else
    launch_one_minus(chi0, n, nfreq, trace, st);
  // the diagonal (of chi0 in a batch, of 1 - chi0 otherwise), for the LU fallback
  launch_diag(chi0, n, nfreq, b.diag, true, st);
  if (mode == MBPT_MODE_MIXED && want_w) {
    // the pair arrays are read as zeros wherever the recursion does not write
    // (padding, above the diagonal blocks); every frequency writes the rest
    for (int i = 0; i < b.npairs; ++i) {
      const PairScratch &q = b.pairs[i];
      const size_t bytes = sizeof(float) * q.np * q.np;
      for (float *f : {q.lr_hi, q.lr_lo, q.ic_hi, q.ic_lo, q.ir_hi, q.ir_lo, q.tt_hi, q.tt_lo})
        if (cudaMemsetAsync(f, 0, bytes, st) != cudaSuccess) return MBPT_ERR_CUDA;
    }
  }
  // the inverse streams: FP64 mode's cuBLAS inverse on the side stream only
  const int nsides = mode == MBPT_MODE_MIXED ? b.npairs : 1;
  auto side_of = [&](int i) { return i == 0 ? pp->side : pp->isides[i - 1]; };
  bool side_used[kMaxInverseStreams] = {};
  if (batched) {
    if (cudaMemsetAsync(b.info, 0, sizeof(int) * nfreq, st) != cudaSuccess) return MBPT_ERR_CUDA;
    // groups of frequencies on their own streams (four by default, each of
    // at least kBatchedCholMin frequencies): one
    // group's DGEMMs fill the GPU while another's diagonal blocks (one CTA
    // per matrix) are factorised
    auto stream_of = [&](int g) { return g == 0 ? st : (g == 1 ? pp->fac2 : pp->xs[g - 2]); };
    auto blas_of = [&](int g) { return g == 0 ? h.blas : (g == 1 ? pp->blas2 : pp->xb[g - 2]); };
    auto join_of = [&](int g) { return g == 1 ? pp->join2 : pp->xj[g - 2]; };
    // waves (MBPT_DYSON_WAVES=2): the frequencies factorised in two halves one
    // after the other on the same streams, the tensor-core inverses of the
    // first half (on the side stream, issued as soon as its factors are done)
    // running beside the second half's FP64 factorisation. Off by default:
    // at naux 7200, 24 frequencies it measured 155.6 ms against 154.0 ms for
    // one wave (the overlap does not pay for the smaller batches)
    const char *wenv = std::getenv("MBPT_DYSON_WAVES");
    const int want_waves = wenv ? std::max(1, std::atoi(wenv)) : 1;
    const int waves = (want_w && nfreq >= 2 * kBatchedCholMin) ? std::min(want_waves, 2) : 1;
    int G = 1;
    for (int w = 0; w < waves; ++w) {
      const int n_w = nfreq * (w + 1) / waves - nfreq * w / waves;
      G = std::max(G, std::min(pp->groups, n_w / kBatchedCholMin));
    }
    if (G > 1 && cudaEventRecord(pp->fork, st) != cudaSuccess) return MBPT_ERR_CUDA;
    for (int g = 1; g < G; ++g)
      if (cudaStreamWaitEvent(stream_of(g), pp->fork, 0) != cudaSuccess) return MBPT_ERR_CUDA;
    int rc0 = MBPT_OK;
    for (int w = 0; w < waves && !rc0; ++w) {
      const int w0 = nfreq * w / waves, nw = nfreq * (w + 1) / waves - w0;
      const int Gw = std::max(1, std::min(G, nw / kBatchedCholMin));
      for (int g = 0; g < Gw && !rc0; ++g) {
        const int f0 = w0 + static_cast<int>(static_cast<int64_t>(nw) * g / Gw);
        const int f1 = w0 + static_cast<int>(static_cast<int64_t>(nw) * (g + 1) / Gw);
        cudaStream_t gs = stream_of(g);
        OzakiChol oz;
        if (b.oz_planes) {
          // this group's frequencies own a contiguous share of each buffer
          oz.planes = b.oz_planes + ozaki_planes_bytes(n, f0, b.oz_slices);
          oz.scale = b.oz_scale + static_cast<int64_t>(f0) * n;
          oz.rowsq = b.oz_rowsq + static_cast<int64_t>(f0) * n;
          oz.slices = b.oz_slices;
          oz.err = err;
        }
        rc0 = chol_batched(chi0 + f0 * n * n, n, f1 - f0, b.info + f0,
                           b.chol_P + static_cast<int64_t>(f0) * n * kCholNb,
                           b.chol_Linv + static_cast<int64_t>(f0) * kCholNb * kCholNb,
                           blas_of(g), gs, static_cast<int64_t>(nfreq) * kCholNb * kCholNb,
                           &oz, true);
        if (rc0) break;
        // this group's log-determinants, info words and events on its own stream
        launch_logdet_diag(chi0 + f0 * n * n, n, f1 - f0, logdet + f0, gs);
        if (!deferred && cudaMemcpyAsync(pp->info + f0, b.info + f0, sizeof(int) * (f1 - f0),
                                         cudaMemcpyDeviceToHost, gs) != cudaSuccess)
          rc0 = MBPT_ERR_CUDA;
        for (int f = f0; f < f1 && !rc0; ++f)
          if (cudaEventRecord(pp->ev[f], gs) != cudaSuccess) rc0 = MBPT_ERR_CUDA;
      }
    }
    for (int g = 1; g < G; ++g)
      if (cudaEventRecord(join_of(g), stream_of(g)) != cudaSuccess ||
          cudaStreamWaitEvent(st, join_of(g), 0) != cudaSuccess)
        return MBPT_ERR_CUDA;
    if (rc0) return rc0;
  }
  const int nfac = nfreq > 1 && !batched ? pp->nfac : 1;
  if (nfac == 2 && (cudaEventRecord(pp->fork, st) != cudaSuccess ||
                    cudaStreamWaitEvent(pp->fac2, pp->fork, 0) != cudaSuccess))
    return MBPT_ERR_CUDA;
  auto factor = [&](int f) -> int {
    if (batched) return MBPT_OK;
    double *m = chi0 + f * n * n;
    const bool second = nfac == 2 && (f & 1);
    cudaStream_t fs = second ? pp->fac2 : st;
    if (cusolverDnDpotrf(second ? pp->solver2 : h.solver, CUBLAS_FILL_MODE_LOWER, ni, m, ni,
                         second ? b.work2 : b.work, b.lwork,
                         b.info + f) != CUSOLVER_STATUS_SUCCESS)
      return MBPT_ERR_CUDA;
    // log det from the factor's diagonal before the inverse overwrites it
    // (replaced below where the factorisation failed)
    launch_logdet_diag(m, n, 1, logdet + f, fs);
    if (cudaMemcpyAsync(pp->info + f, b.info + f, sizeof(int), cudaMemcpyDeviceToHost, fs) !=
            cudaSuccess ||
        cudaEventRecord(pp->ev[f], fs) != cudaSuccess)
      return MBPT_ERR_CUDA;
    return MBPT_OK;
  };
  bool bad = false;
  int rc = MBPT_OK;
  for (int f = 0; f < nfac && f < nfreq && rc == MBPT_OK; ++f) rc = factor(f);
  for (int f = 0; f < nfreq && rc == MBPT_OK; ++f) {
    if (f + nfac < nfreq && (rc = factor(f + nfac)) != MBPT_OK) break;
    if (!deferred && cudaEventSynchronize(pp->ev[f]) != cudaSuccess) {
      rc = MBPT_ERR_CUDA;
      break;
    }
    const int inf = deferred ? 0 : pp->info[f];
    if (info_host && !deferred) info_host[f] = inf;
    if (sign_host) sign_host[f] = 1;
    double *m = chi0 + f * n * n;
    if (inf == 0) {
      if (want_w) {
        const int si = f % nsides;
        cudaStream_t ss = side_of(si);
        side_used[si] = true;
        if (cudaStreamWaitEvent(ss, pp->ev[f], 0) != cudaSuccess) {
          rc = MBPT_ERR_CUDA;
          break;
        }
        Handles hs{pp->blas_side, h.solver};
        bool full = false;
        rc = spd_inverse_from_factor(
            hs, m, n, b.T, b.rhs, mode == MBPT_MODE_MIXED ? &b.pairs[si] : nullptr, err, &full,
            ss, batched ? b.chol_Linv + static_cast<int64_t>(f) * kCholNb * kCholNb : nullptr,
            static_cast<int64_t>(nfreq) * kCholNb * kCholNb);
        if (rc) break;
        if (!full) launch_symmetrize_minus_identity(m, n, 1, ss);
      }
      continue;
    }
    // not positive definite: drain every stream (the LU shares the scratch),
    // restore 1 - chi0 from its untouched triangle, then LU for log|det| (and
    // the inverse), as the reference's slogdet/inv
    bad = true;
    for (int i = 1; i < nsides; ++i)
      if (cudaStreamSynchronize(side_of(i)) != cudaSuccess) rc = MBPT_ERR_CUDA;
    if (rc || cudaStreamSynchronize(pp->side) != cudaSuccess ||
        (nfac == 2 && cudaStreamSynchronize(pp->fac2) != cudaSuccess) ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      rc = MBPT_ERR_CUDA;
      break;
    }
    launch_mirror_lower_to_upper(m, n, st);
    launch_diag(m, n, 1, b.diag + static_cast<int64_t>(f) * n, false, st);
    // a batch left chi0 in the untouched triangle
    if (batched) launch_one_minus(m, n, 1, nullptr, st);
    if (cusolverDnDgetrf(h.solver, ni, ni, m, ni, b.work, b.piv, b.info + nfreq) !=
        CUSOLVER_STATUS_SUCCESS) {
      rc = MBPT_ERR_CUDA;
      break;
    }
    int sgn = 1;
    int *sgn_dev = b.info + nfreq;
    launch_lu_logdet(m, b.piv, n, logdet + f, sgn_dev, st);
    cudaMemcpyAsync(&sgn, sgn_dev, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (want_w) {
      // inverse from the LU factor: solve against the identity, minus I
      launch_identity(b.rhs, n, st);
      if (cusolverDnDgetrs(h.solver, CUBLAS_OP_N, ni, ni, m, ni, b.piv, b.rhs, ni,
                           b.info + nfreq) != CUSOLVER_STATUS_SUCCESS) {
        rc = MBPT_ERR_CUDA;
        break;
      }
      cudaMemcpyAsync(m, b.rhs, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, st);
      launch_minus_identity(m, n, st);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      rc = MBPT_ERR_CUDA;
      break;
    }
    if (sign_host) sign_host[f] = sgn;
  }
  for (int i = 0; i < nsides; ++i) {
    if (!side_used[i]) continue;
    cudaEvent_t j = i == 0 ? pp->join : pp->ijoin[i - 1];
    cudaEventRecord(j, side_of(i));
    cudaStreamWaitEvent(st, j, 0);
  }
  if (nfac == 2) {
    cudaEventRecord(pp->join2, pp->fac2);
    cudaStreamWaitEvent(st, pp->join2, 0);
  }
  if (rc) return rc;
  if (deferred && cudaMemcpyAsync(info_dev_out, b.info, sizeof(int) * nfreq,
                                  cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MBPT_ERR_CUDA;
  if (cudaGetLastError() != cudaSuccess) return MBPT_ERR_CUDA;
  return bad ? MBPT_ERR_NOT_SPD : MBPT_OK;
}

// -------------------------------------------------------------------- Sigma
struct SigmaBufs {
  // fp64
  double *U, *Zt, *G, *Xo_s, *Xv_s, *Xs, *R;
  // mixed
  bf16 *D_hi, *D_lo, *W_hi, *W_lo, *U_hi, *U_lo, *Yo_hi, *Yo_lo, *Yv_hi, *Yv_lo, *Hl_hi,
      *Hl_lo, *Hg_hi, *Hg_lo, *XsT_hi, *XsT_lo;
  float *xs, *Zf;
  double *sig;
};

int64_t pad_states(int nstates) { return round_up(nstates, 128); }

SigmaBufs carve_sigma(Arena &ar, const Dims &d, int ntau, int nstates, int mode) {
  SigmaBufs b{};
  if (fp64_mode(mode)) {
    b.U = ar.take<double>(d.M * d.naux);
    b.Zt = ar.take<double>(d.M * d.M);
    b.G = ar.take<double>(d.M * d.M);
    b.Xo_s = ar.take<double>(d.M * d.nocc);
    b.Xv_s = ar.take<double>(d.M * d.nv);
    b.Xs = ar.take<double>(d.M * static_cast<int64_t>(nstates));
    b.R = ar.take<double>(d.M * static_cast<int64_t>(nstates));
  } else {
    const int64_t Sp = pad_states(nstates);
    b.D_hi = ar.take<bf16>(d.Mp * d.Ap);
    b.D_lo = ar.take<bf16>(d.Mp * d.Ap);
    b.W_hi = ar.take<bf16>(d.Ap * d.Ap);
    b.W_lo = ar.take<bf16>(d.Ap * d.Ap);
    b.U_hi = ar.take<bf16>(d.Mp * d.Ap);
    b.U_lo = ar.take<bf16>(d.Mp * d.Ap);
    b.Yo_hi = ar.take<bf16>(d.Mp * d.Ko);
    b.Yo_lo = ar.take<bf16>(d.Mp * d.Ko);
    b.Yv_hi = ar.take<bf16>(d.Mp * d.Kv);
    b.Yv_lo = ar.take<bf16>(d.Mp * d.Kv);
    b.Hl_hi = ar.take<bf16>(d.Mp * d.Mp);
    b.Hl_lo = ar.take<bf16>(d.Mp * d.Mp);
    b.Hg_hi = ar.take<bf16>(d.Mp * d.Mp);
    b.Hg_lo = ar.take<bf16>(d.Mp * d.Mp);
    b.XsT_hi = ar.take<bf16>(Sp * d.Mp);
    b.XsT_lo = ar.take<bf16>(Sp * d.Mp);
    b.xs = ar.take<float>(d.Mp * Sp);
    b.Zf = ar.take<float>(d.Mp * d.Mp);
    b.sig = ar.take<double>(2 * static_cast<int64_t>(ntau) * Sp);
  }
  return b;
}

int sigma_run(const double *X, const Dims &d, const double *eps, double mu, const double *D,
              const double *Wt, const double *tau, int ntau, const int64_t *states,
              int nstates, int mode, double *branch, Arena &ar, int *err, cudaStream_t st) {
  SigmaBufs b = carve_sigma(ar, d, ntau, nstates, mode);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  const int64_t a2 = d.naux * d.naux;
  const int64_t S = nstates;
  if (fp64_mode(mode)) {
    cublasHandle_t h = handles(st).blas;
    launch_gather_cols_f64(X, d.M, d.n, states, S, b.Xs, st);
    for (int k = 0; k < ntau; ++k) {
      // Zt = D Wt D^T (MBPTcode imaginary_time.py:508, :513); Wt = I without Wt
      if (Wt && !gemm_mode(mode, h, false, false, d.M, d.naux, d.naux, 1.0, D, d.naux,
                           Wt + k * a2, d.naux, 0.0, b.U, d.naux))
        return MBPT_ERR_CUDA;
      if ((Wt || k == 0) && !gemm_mode(mode, h, false, true, d.M, d.M, d.naux, 1.0,
                                       Wt ? b.U : D, d.naux, D, d.naux, 0.0, b.Zt, d.M, true))
        return MBPT_ERR_CUDA;
      launch_scaled_branches(X, d.M, d.n, d.nocc, eps, mu, tau[k], 1.0, b.Xo_s, b.Xv_s, st);
      double *out_l = branch + static_cast<int64_t>(k) * S;
      double *out_g = branch + static_cast<int64_t>(ntau + k) * S;
      // lesser branch: G_occ o Zt contracted with X_s on both sides
      if (!gemm_mode(mode, h, false, true, d.M, d.M, d.nocc, 1.0, b.Xo_s, d.nocc, X, d.n, 0.0,
                     b.G, d.M))
        return MBPT_ERR_CUDA;
      launch_hadamard(b.G, b.Zt, d.M * d.M, st);
      if (!gemm_mode(mode, h, false, false, d.M, S, d.M, 1.0, b.G, d.M, b.Xs, S, 0.0, b.R, S))
        return MBPT_ERR_CUDA;
      cudaMemsetAsync(out_l, 0, sizeof(double) * S, st);
      launch_rowdot(b.R, S, b.Xs, S, d.M, S, 1.0, out_l, st);
      // greater branch, with its minus sign
      if (!gemm_mode(mode, h, false, true, d.M, d.M, d.nv, 1.0, b.Xv_s, d.nv, X + d.nocc, d.n,
                     0.0, b.G, d.M))
        return MBPT_ERR_CUDA;
      launch_hadamard(b.G, b.Zt, d.M * d.M, st);
      if (!gemm_mode(mode, h, false, false, d.M, S, d.M, 1.0, b.G, d.M, b.Xs, S, 0.0, b.R, S))
        return MBPT_ERR_CUDA;
      cudaMemsetAsync(out_g, 0, sizeof(double) * S, st);
      launch_rowdot(b.R, S, b.Xs, S, d.M, S, -1.0, out_g, st);
    }
  } else {
    const int64_t Sp = pad_states(nstates);
    launch_split_pad<double>(D, d.M, d.naux, d.naux, 1.f, b.D_hi, b.D_lo, d.Ap, d.Mp, d.Ap,
                             false, st);
    launch_gather_cols_f32(X, d.M, d.n, states, S, b.xs, Sp, d.Mp, st);
    launch_gather_cols_split_t(X, d.M, d.n, states, S, b.XsT_hi, b.XsT_lo, d.Mp, Sp, d.Mp, st);
    cudaMemsetAsync(b.sig, 0, sizeof(double) * 2 * ntau * Sp, st);
    SplitMat Dm{b.D_hi, b.D_lo, d.Mp, d.Ap, d.Ap};
    SplitMat Wm{b.W_hi, b.W_lo, d.Ap, d.Ap, d.Ap};
    SplitMat Um{b.U_hi, b.U_lo, d.Mp, d.Ap, d.Ap};
    SplitMat Yo{b.Yo_hi, b.Yo_lo, d.Mp, d.Ko, d.Ko}, Yv{b.Yv_hi, b.Yv_lo, d.Mp, d.Kv, d.Kv};
    SplitMat Hl{b.Hl_hi, b.Hl_lo, d.Mp, d.Mp, d.Mp}, Hg{b.Hg_hi, b.Hg_lo, d.Mp, d.Mp, d.Mp};
    SplitMat XsT{b.XsT_hi, b.XsT_lo, Sp, d.Mp, d.Mp};
    for (int k = 0; k < ntau; ++k) {
      launch_prep_branches(X, d.M, d.n, d.nocc, eps, mu, tau[k], b.Yo_hi, b.Yo_lo, d.Ko,
                           b.Yv_hi, b.Yv_lo, d.Kv, d.Mp, st);
      umma::EpiArgs e;
      int rc = MBPT_OK;
      if (Wt) {
        // U = D Wt (Wt symmetric); without Wt, W = I and U = D
        launch_split_pad<double>(Wt + k * a2, d.naux, d.naux, d.naux, 1.f, b.W_hi, b.W_lo,
                                 d.Ap, d.Ap, d.Ap, false, st);
        e.out0_hi = b.U_hi;
        e.out0_lo = b.U_lo;
        e.ld_out = d.Ap;
        rc = gemm_split(umma::EPI_SPLIT, 1, &Dm, &Wm, d.Mp, d.Ap, e, err, st);
        if (rc) return rc;
      }
      // Zt = U D^T (= D W D^T, symmetric) whole in FP32: upper 256 x 256 tiles
      // on CTA pairs, mirrored by the epilogue, its K = naux sum drained
      e = umma::EpiArgs();
      e.outf = b.Zf;
      e.ld_outf = d.Mp;
      e.alpha = 1.f;
      rc = gemm_split(umma::EPI_F32, 1, Wt ? &Um : &Dm, &Dm, d.Mp, d.Mp, e, err, st,
                      umma::BAND_UPPER);
      if (rc) return rc;
      // G_occ, G_virt (short K) -> H< = G_occ o Zt, H> = G_virt o Zt; all four
      // symmetric: upper tiles, mirrored by the epilogue
      e = umma::EpiArgs();
      e.out0_hi = b.Hl_hi;
      e.out0_lo = b.Hl_lo;
      e.out1_hi = b.Hg_hi;
      e.out1_lo = b.Hg_lo;
      e.ld_out = d.Mp;
      e.zt = b.Zf;
      e.ld_zt = d.Mp;
      SplitMat A2g[2] = {Yo, Yv};
      rc = gemm_split(umma::EPI_SIGMA_HZ, 2, A2g, A2g, d.Mp, d.Mp, e, err, st,
                      umma::BAND_UPPER);
      if (rc) return rc;
      // branch sums: sum_P X_s[P,p] (H X_s)[P,p]
      e = umma::EpiArgs();
      e.xs = b.xs;
      e.ld_xs = Sp;
      e.sig0 = b.sig + static_cast<int64_t>(k) * Sp;
      e.sig1 = b.sig + static_cast<int64_t>(ntau + k) * Sp;
      SplitMat A2[2] = {Hl, Hg}, B2[2] = {XsT, XsT};
      rc = gemm_split(umma::EPI_ROWDOT2, 2, A2, B2, d.Mp, Sp, e, err, st);
      if (rc) return rc;
    }
    cudaMemcpy2DAsync(branch, sizeof(double) * S, b.sig, sizeof(double) * Sp,
                      sizeof(double) * S, 2 * ntau, cudaMemcpyDeviceToDevice, st);
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// ------------------------------------------------------------- chi0 adjoint
struct BackBufs {
  double *pb, *E, *Xo_s, *Xv_s, *Go, *Gv, *P, *T, *GoX, *GvX;
};

BackBufs carve_back(Arena &ar, const Dims &d) {
  BackBufs b{};
  b.pb = ar.take<double>(d.naux * d.naux);
  b.E = ar.take<double>(d.M * d.naux);
  b.Xo_s = ar.take<double>(d.M * d.nocc);
  b.Xv_s = ar.take<double>(d.M * d.nv);
  b.Go = ar.take<double>(d.M * d.M);
  b.Gv = ar.take<double>(d.M * d.M);
  b.P = ar.take<double>(d.M * d.M);
  b.T = ar.take<double>(d.M * d.M);
  b.GoX = ar.take<double>(d.M * d.nocc);
  b.GvX = ar.take<double>(d.M * d.nv);
  return b;
}

int back_run(const double *pbar, const double *X, const Dims &d, const double *eps, double mu,
             const double *D, const double *tau, int ntau, double *eps_bar, double *X_bar,
             double *D_bar, Arena &ar, cudaStream_t st, int mode) {
  BackBufs b = carve_back(ar, d);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  const int64_t a2 = d.naux * d.naux;
  cudaMemsetAsync(eps_bar, 0, sizeof(double) * d.n, st);
  cudaMemsetAsync(X_bar, 0, sizeof(double) * d.M * d.n, st);
  cudaMemsetAsync(D_bar, 0, sizeof(double) * d.M * d.naux, st);
  for (int k = 0; k < ntau; ++k) {
    // MBPTcode gradients/rpa/space_time_adjoint.py:196-217, one row tile
    launch_sym_half(pbar + k * a2, b.pb, d.naux, st);
    if (!gemm_mode(mode, h, false, false, d.M, d.naux, d.naux, -2.0, D, d.naux, b.pb, d.naux, 0.0,
                  b.E, d.naux))
      return MBPT_ERR_CUDA;
    launch_scaled_branches(X, d.M, d.n, d.nocc, eps, mu, tau[k], 1.0, b.Xo_s, b.Xv_s, st);
    if (!gemm_mode(mode, h, false, true, d.M, d.M, d.nocc, 1.0, b.Xo_s, d.nocc, X, d.n, 0.0, b.Go,
                  d.M) ||
        !gemm_mode(mode, h, false, true, d.M, d.M, d.nv, 1.0, b.Xv_s, d.nv, X + d.nocc, d.n, 0.0,
                  b.Gv, d.M))
      return MBPT_ERR_CUDA;
    launch_hadamard3(b.P, b.Go, b.Gv, d.M * d.M, st);  // Pi
    if (!gemm_mode(mode, h, false, false, d.M, d.naux, d.M, 2.0, b.P, d.M, b.E, d.naux, 1.0, D_bar,
                  d.naux))
      return MBPT_ERR_CUDA;
    // Pi_bar = E D^T (symmetric) and the G branches' adjoints Go_bar =
    // Pi_bar o Gv, Gv_bar = Pi_bar o Go: on the Ozaki product both straight
    // from its epilogue (Pi_bar never stored), else through Pi_bar
    double *go_bar = b.P, *gv_bar = b.T;
    if (mode == MBPT_MODE_FP64_INT8 && d.naux <= kOzakiKChunk) {
      OzakiEpi e;
      e.sym = true;
      e.h1 = b.Gv;
      e.h2 = b.Go;
      e.c2 = gv_bar;
      if (!gemm_ozaki(h, false, true, d.M, d.M, d.naux, 1.0, b.E, d.naux, D, d.naux, 0.0,
                      go_bar, d.M, &e))
        return MBPT_ERR_CUDA;
    } else {
      if (!dgemm_rm(h, false, true, d.M, d.M, d.naux, 1.0, b.E, d.naux, D, d.naux, 0.0, b.P,
                    d.M))
        return MBPT_ERR_CUDA;
      launch_hadamard3(gv_bar, b.P, b.Go, d.M * d.M, st);
      go_bar = b.Go;  // G_occ is not read again at this tau point
      launch_hadamard3(go_bar, b.P, b.Gv, d.M * d.M, st);
    }
    if (!gemm_mode(mode, h, false, false, d.M, d.nocc, d.M, 1.0, go_bar, d.M, X, d.n, 0.0, b.GoX,
                  d.nocc) ||
        !gemm_mode(mode, h, false, false, d.M, d.nv, d.M, 1.0, gv_bar, d.M, X + d.nocc, d.n, 0.0,
                  b.GvX, d.nv))
      return MBPT_ERR_CUDA;
    launch_xbar_update(b.GoX, b.GvX, X, d.M, d.n, d.nocc, eps, mu, tau[k], X_bar, eps_bar, st);
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// ------------------------------------------------------- self-energy adjoint
struct SigBackBufs {
  double *Xo_s, *Xv_s, *Go, *Gv, *Zt, *Al, *Ag, *U, *Xs, *Xl, *Xg, *T1, *GoX, *GvX;
};

SigBackBufs carve_sigma_back(Arena &ar, const Dims &d, int64_t S) {
  SigBackBufs b{};
  b.Xo_s = ar.take<double>(d.M * d.nocc);
  b.Xv_s = ar.take<double>(d.M * d.nv);
  for (double **m : {&b.Go, &b.Gv, &b.Zt, &b.Al, &b.Ag}) *m = ar.take<double>(d.M * d.M);
  b.U = ar.take<double>(d.M * d.naux);
  for (double **m : {&b.Xs, &b.Xl, &b.Xg, &b.T1}) *m = ar.take<double>(d.M * S);
  b.GoX = ar.take<double>(d.M * d.nocc);
  b.GvX = ar.take<double>(d.M * d.nv);
  return b;
}

// The reverse of the states' self-energy branch sums over every tau point,
// in the grid-space form of the forward: Sigma^<_s(tau) = x_s^T (Go o Zt) x_s,
// Sigma^>_s(tau) = -x_s^T (Gv o Zt) x_s with Zt = D Wt(tau) D^T and x_s the
// state's column of X. For the branch adjoints sl, sg of one tau point, with
// Al = sum_s sl_s x_s x_s^T and Ag = sum_s sg_s x_s x_s^T:
//   x_s_bar  = 2 [(Go o Zt) x_s sl_s - (Gv o Zt) x_s sg_s],
//   Go_bar   = Zt o Al,   Gv_bar = -Zt o Ag    (then the G branches' reverse),
//   Zt_bar   = Go o Al - Gv o Ag,
//   Wt_bar   = D^T Zt_bar D,   D_bar += 2 Zt_bar D Wt.
// It is the same derivative as MBPTcode gradients/rpa/space_time_adjoint.py:836-856
// (written there on the three-index slices B_p = D^T diag(x_p) X), and
// :866-871 for the bra slices' share of X_bar and D_bar.
int sigma_back_run(const double *X, const Dims &d, const double *eps, double mu,
                   const double *D, const double *tau, int ntau, const double *Wt,
                   const int64_t *states, int64_t S, const double *sl_bar,
                   const double *sg_bar, double *eps_bar, double *X_bar, double *D_bar,
                   double *Wt_bar, Arena &ar, cudaStream_t st, int mode) {
  SigBackBufs b = carve_sigma_back(ar, d, S);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  const int64_t a2 = d.naux * d.naux, M = d.M, A = d.naux;
  cudaMemsetAsync(eps_bar, 0, sizeof(double) * d.n, st);
  cudaMemsetAsync(X_bar, 0, sizeof(double) * M * d.n, st);
  cudaMemsetAsync(D_bar, 0, sizeof(double) * M * A, st);
  for (int k = 0; k < ntau; ++k) {
    const double *Wk = Wt + k * a2;
    launch_scaled_branches(X, M, d.n, d.nocc, eps, mu, tau[k], 1.0, b.Xo_s, b.Xv_s, st);
    launch_sigma_back_gather(X, M, d.n, states, S, sl_bar + k * S, sg_bar + k * S, b.Xs, b.Xl,
                             b.Xg, st);
    if (!gemm_mode(mode, h, false, true, M, M, d.nocc, 1.0, b.Xo_s, d.nocc, X, d.n, 0.0, b.Go, M) ||
        !gemm_mode(mode, h, false, true, M, M, d.nv, 1.0, b.Xv_s, d.nv, X + d.nocc, d.n, 0.0, b.Gv,
                  M) ||
        !gemm_mode(mode, h, false, false, M, A, A, 1.0, D, A, Wk, A, 0.0, b.U, A) ||
        !gemm_mode(mode, h, false, true, M, M, A, 1.0, b.U, A, D, A, 0.0, b.Zt, M, true) ||
        !gemm_mode(mode, h, false, true, M, M, S, 1.0, b.Xl, S, b.Xs, S, 0.0, b.Al, M) ||
        !gemm_mode(mode, h, false, true, M, M, S, 1.0, b.Xg, S, b.Xs, S, 0.0, b.Ag, M))
      return MBPT_ERR_CUDA;
    // Go -> L = Go o Zt, Gv -> H = Gv o Zt, Zt -> Zt_bar, Al -> Go_bar, Ag -> Gv_bar
    launch_sigma_back_hadamard(b.Go, b.Gv, b.Zt, b.Al, b.Ag, M * M, st);
    if (!gemm_mode(mode, h, false, false, M, S, M, 1.0, b.Go, M, b.Xl, S, 0.0, b.T1, S) ||
        !gemm_mode(mode, h, false, false, M, S, M, -1.0, b.Gv, M, b.Xg, S, 1.0, b.T1, S))
      return MBPT_ERR_CUDA;
    launch_scatter_cols(b.T1, M, S, states, 2.0, X_bar, d.n, st);
    if (!gemm_mode(mode, h, false, false, M, d.nocc, M, 1.0, b.Al, M, X, d.n, 0.0, b.GoX, d.nocc) ||
        !gemm_mode(mode, h, false, false, M, d.nv, M, 1.0, b.Ag, M, X + d.nocc, d.n, 0.0, b.GvX,
                  d.nv))
      return MBPT_ERR_CUDA;
    launch_xbar_update(b.GoX, b.GvX, X, M, d.n, d.nocc, eps, mu, tau[k], X_bar, eps_bar, st);
    // U <- Zt_bar D, then Wt_bar = D^T U and D_bar += 2 U Wt (Zt_bar and Wt symmetric)
    if (!gemm_mode(mode, h, false, false, M, A, M, 1.0, b.Zt, M, D, A, 0.0, b.U, A) ||
        !gemm_mode(mode, h, true, false, A, A, M, 1.0, D, A, b.U, A, 0.0, Wt_bar + k * a2, A) ||
        !gemm_mode(mode, h, false, false, M, A, A, 2.0, b.U, A, Wk, A, 1.0, D_bar, A))
      return MBPT_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// chi0_bar_f = W_f W_bar_f W_f in place over W_bar, W_f = I + (W - I)_f:
// the reverse of the Dyson step W = [1 - chi0]^-1 (W symmetric), as MBPTcode
// gradients/rpa/space_time_adjoint.py:679-685
int dyson_back_run(const double *wmi, double *wbar, int64_t n, int nfreq, Arena &ar,
                   cudaStream_t st, int mode) {
  double *T = ar.take<double>(n * n);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  const size_t bytes = sizeof(double) * n * n;
  for (int f = 0; f < nfreq; ++f) {
    const double *Wm = wmi + f * n * n;
    double *B = wbar + f * n * n;
    // T = B + Wm B; B <- T + T Wm
    if (cudaMemcpyAsync(T, B, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        !gemm_mode(mode, h, false, false, n, n, n, 1.0, Wm, n, B, n, 1.0, T, n) ||
        cudaMemcpyAsync(B, T, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        !gemm_mode(mode, h, false, false, n, n, n, 1.0, T, n, Wm, n, 1.0, B, n))
      return MBPT_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t count(void (*f)(Arena &)) {
  Arena ar;
  ar.counting = true;
  f(ar);
  return ar.used + 1024;
}

Arena arena(void *ws, size_t bytes) {
  Arena ar;
  ar.base = reinterpret_cast<uint8_t *>(ws);
  ar.size = bytes;
  if (reinterpret_cast<uintptr_t>(ws) & 1023) {
    const size_t skip = 1024 - (reinterpret_cast<uintptr_t>(ws) & 1023);
    ar.base += skip;
    ar.size = bytes > skip ? bytes - skip : 0;
  }
  return ar;
}

}  // namespace
}  // namespace mbpt

using namespace mbpt;

extern "C" {

int mbpt_abi_version(void) { return kAbiVersion; }

const char *mbpt_status_string(int s) {
  switch (s) {
    case MBPT_OK: return "ok";
    case MBPT_ERR_SHAPE: return "inconsistent or unsupported sizes";
    case MBPT_ERR_NOT_SPD: return "1 - chi0 is not positive definite at some frequency";
    case MBPT_ERR_NONFINITE: return "non-finite value";
    case MBPT_ERR_NO_ROOT: return "quasiparticle equation without a root";
    case MBPT_ERR_TIMEOUT: return "a bounded device-side wait ran out";
    case MBPT_ERR_CUDA: return "CUDA runtime or library error";
    case MBPT_ERR_WORKSPACE: return "workspace too small";
    case MBPT_ERR_UNSUPPORTED: return "unsupported device or option";
    default: return "unknown status";
  }
}

long long mbpt_launch_count(void) { return g_launches.load(); }

int mbpt_wait_selftest(int arrive, int limit_us, int *err_dev, void *stream) {
  return wait_selftest(arrive, limit_us, err_dev, S(stream));
}

int mbpt_gemm_timing(int enable, double *total_ms, long long *launches) {
  return gemm_timing(enable, total_ms, launches);
}

int mbpt_energy_sum(const double *logdet, const double *trace, const double *w, int nfreq,
                    double *e_c, void *stream) {
  if (nfreq < 1) return MBPT_ERR_SHAPE;
  launch_energy_sum(logdet, trace, w, nfreq, e_c, S(stream));
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int mbpt_device_supported(int device) {
  // two attributes, not cudaGetDeviceProperties (which takes milliseconds)
  int major = 0, minor = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device) != cudaSuccess)
    return 0;
  return major == 10 && minor == 0 ? 1 : 0;
}

size_t mbpt_chi0_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux, int ntau,
                                 int mode) {
  Dims d(M, norb, nocc, naux);
  Arena ar;
  ar.counting = true;
  carve_chi0(ar, d, ntau, 34, mode, true);
  return ar.used + 2048;
}

int mbpt_chi0_sweep(const double *X, int64_t M, int64_t norb, int64_t nocc, const double *eps,
                    double mu, const double *D, int64_t naux, const double *tau, int ntau,
                    const double *cw, int nfreq, int mode, double *chi0, double *proj,
                    void *ws, size_t ws_bytes, int *err, void *stream) {
  Dims d(M, norb, nocc, naux);
  if (!d.ok() || ntau < 1 || nfreq < 1 || ntau > 34 || nfreq > 34) return MBPT_ERR_SHAPE;
  if (!valid_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  Arena ar = arena(ws, ws_bytes);
  return chi0_run(X, d, eps, mu, D, tau, ntau, cw, nfreq, mode, chi0, proj, ar, err, S(stream));
}

size_t mbpt_dyson_workspace_bytes(int64_t naux, int nfreq, int mode) {
  Arena ar;
  ar.counting = true;
  carve_dyson(ar, naux, nfreq, mode);
  return ar.used + 2048;
}

int mbpt_dyson(double *chi0, int64_t naux, int nfreq, int want_w, int mode, double *logdet,
               double *trace, int *info_host, int *sign_host, void *ws, size_t ws_bytes,
               int *err, void *stream) {
  if (naux < 1 || nfreq < 1) return MBPT_ERR_SHAPE;
  if (!valid_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  Arena ar = arena(ws, ws_bytes);
  return dyson_run(chi0, naux, nfreq, want_w, logdet, trace, info_host, sign_host, ar,
                   S(stream), mode, err);
}

int mbpt_dyson_deferred(double *chi0, int64_t naux, int nfreq, int want_w, int mode,
                        double *logdet, double *trace, int *info_dev, void *ws, size_t ws_bytes,
                        int *err, void *stream) {
  if (naux < 1 || nfreq < 1 || !info_dev) return MBPT_ERR_SHAPE;
  if (!valid_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  Arena ar = arena(ws, ws_bytes);
  return dyson_run(chi0, naux, nfreq, want_w, logdet, trace, nullptr, nullptr, ar, S(stream),
                   mode, err, info_dev);
}

size_t mbpt_rpa_energy_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux,
                                       int ntau, int nfreq, int mode) {
  Dims d(M, norb, nocc, naux);
  Arena ar;
  ar.counting = true;
  ar.take<double>(static_cast<size_t>(nfreq) * naux * naux);  // chi0
  ar.take<double>(34);                                         // logdet
  ar.take<double>(34);                                         // trace
  ar.take<double>(34);                                         // weights
  Arena a2 = ar;
  carve_chi0(ar, d, ntau, nfreq, mode, true);
  carve_dyson(a2, naux, nfreq);
  return (ar.used > a2.used ? ar.used : a2.used) + 4096;
}

int mbpt_rpa_energy(const double *X, int64_t M, int64_t norb, int64_t nocc, const double *eps,
                    double mu, const double *D, int64_t naux, const double *tau, int ntau,
                    const double *cw, const double *ow, int nfreq, int mode, double *e_c,
                    double *proj, int *info_host, void *ws, size_t ws_bytes, int *err,
                    void *stream) {
  Dims d(M, norb, nocc, naux);
  if (!d.ok() || ntau < 1 || nfreq < 1 || ntau > 34 || nfreq > 34) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  double *chi0 = ar.take<double>(static_cast<size_t>(nfreq) * naux * naux);
  double *logdet = ar.take<double>(34);
  double *trace = ar.take<double>(34);
  double *w = ar.take<double>(34);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  Arena rest = ar;
  int rc = chi0_run(X, d, eps, mu, D, tau, ntau, cw, nfreq, mode, chi0, proj, rest, err, st);
  if (rc) return rc;
  rest = ar;
  rc = dyson_run(chi0, naux, nfreq, 0, logdet, trace, info_host, nullptr, rest, st);
  if (rc && rc != MBPT_ERR_NOT_SPD) return rc;
  cudaMemcpyAsync(w, ow, sizeof(double) * nfreq, cudaMemcpyHostToDevice, st);
  launch_energy_sum(logdet, trace, w, nfreq, e_c, st);
  if (cudaGetLastError() != cudaSuccess) return MBPT_ERR_CUDA;
  return rc;
}

int mbpt_transform(const double *in, int K, int64_t n, const double *w_dev, int J,
                   double *out, void *stream) {
  if (K < 1 || J < 1 || K > 34 || J > 34 || n < 1) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  launch_transform<double>(in, n * n, n, n, n, w_dev, J, K, out, n * n, n, st);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int mbpt_transform_acc(const double *in, int K, int64_t n, const double *w_dev, int J,
                       double *out, void *stream) {
  if (K < 1 || J < 1 || K > 34 || J > 34 || n < 1) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  launch_transform_acc(in, n * n, n, n, n, w_dev, J, K, out, n * n, n, st);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t mbpt_sigma_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux, int ntau,
                                  int nstates, int mode) {
  Dims d(M, norb, nocc, naux);
  Arena ar;
  ar.counting = true;
  carve_sigma(ar, d, ntau, nstates, mode);
  return ar.used + 2048;
}

int mbpt_sigma_branch_sums(const double *X, int64_t M, int64_t norb, int64_t nocc,
                           const double *eps, double mu, const double *D, int64_t naux,
                           const double *Wt, const double *tau, int ntau,
                           const int64_t *states, int nstates, int mode, double *branch,
                           void *ws, size_t ws_bytes, int *err, void *stream) {
  Dims d(M, norb, nocc, naux);
  if (!d.ok() || ntau < 1 || nstates < 1) return MBPT_ERR_SHAPE;
  if (!valid_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  Arena ar = arena(ws, ws_bytes);
  return sigma_run(X, d, eps, mu, D, Wt, tau, ntau, states, nstates, mode, branch, ar, err,
                   S(stream));
}

int mbpt_sigma_frequency(const double *branch, int ntau, int nstates, const double *C_dev,
                         const double *S_dev, int npade, double *sigma, void *stream) {
  if (ntau < 1 || nstates < 1 || npade < 1) return MBPT_ERR_SHAPE;
  launch_sigma_frequency(branch, ntau, nstates, C_dev, S_dev, npade, sigma, S(stream));
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int mbpt_qp_solve(const double *sigma, const double *pade_freq_host, int npade,
                  const double *eps_anchor, const double *xc, const int64_t *states,
                  int nstates, int64_t nocc, double mu, int greedy, const double *warm,
                  double *roots, double *z, int *flags, int *evals, void *ws, size_t ws_bytes,
                  void *stream) {
  if (npade < 2 || npade > 32) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  double *pf = ar.take<double>(npade);
  if (!pf || ar.overflow()) return MBPT_ERR_WORKSPACE;
  cudaMemcpyAsync(pf, pade_freq_host, sizeof(double) * npade, cudaMemcpyHostToDevice, st);
  return launch_pade_qp(sigma, pf, npade, eps_anchor, xc, states, nstates, nocc, mu, greedy,
                        warm, roots, z, flags, evals, st);
}

int mbpt_pade_eval(const double *sigma, const double *pade_freq_host, int npade,
                   const int64_t *states, int nstates, int64_t nocc, double mu, int greedy,
                   const double *query, int nq, double *out, void *ws, size_t ws_bytes,
                   void *stream) {
  if (npade < 2 || npade > 32) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  double *pf = ar.take<double>(npade);
  if (!pf || ar.overflow()) return MBPT_ERR_WORKSPACE;
  cudaMemcpyAsync(pf, pade_freq_host, sizeof(double) * npade, cudaMemcpyHostToDevice, st);
  return launch_pade_eval(sigma, pf, npade, states, nstates, nocc, mu, greedy, query, nq, out,
                          st);
}

size_t mbpt_chi0_backward_workspace_bytes(int64_t M, int64_t norb, int64_t nocc, int64_t naux,
                                          int mode) {
  (void)mode;
  Dims d(M, norb, nocc, naux);
  Arena ar;
  ar.counting = true;
  carve_back(ar, d);
  return ar.used + 2048;
}

int mbpt_chi0_backward(const double *pbar, const double *X, int64_t M, int64_t norb,
                       int64_t nocc, const double *eps, double mu, const double *D,
                       int64_t naux, const double *tau, int ntau, int mode, double *eps_bar,
                       double *X_bar, double *D_bar, void *ws, size_t ws_bytes, int *err,
                       void *stream) {
  (void)err;
  Dims d(M, norb, nocc, naux);
  if (!d.ok() || ntau < 1) return MBPT_ERR_SHAPE;
  if (!fp64_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  Arena ar = arena(ws, ws_bytes);
  return back_run(pbar, X, d, eps, mu, D, tau, ntau, eps_bar, X_bar, D_bar, ar, S(stream),
                  mode);
}

// The full AO self-energy's scratch. FP64 modes: X_mo, the scaled branches,
// G_occ, G_virt, Zt, U = D W(tau) and R; mixed: X_mo and the split (BF16
// pair) operands of the engine's products.
struct SigmaAoBufs {
  double *Xmo = nullptr, *Xs = nullptr, *Go = nullptr, *Gv = nullptr, *Zt = nullptr,
         *U = nullptr, *R = nullptr;
  bf16 *D_hi, *D_lo, *W_hi, *W_lo, *U_hi, *U_lo, *Yo_hi, *Yo_lo, *Yv_hi, *Yv_lo, *Hl_hi,
      *Hl_lo, *Hg_hi, *Hg_lo, *XaT_hi, *XaT_lo, *RT_hi, *RT_lo;
  float *Zf = nullptr;
};

SigmaAoBufs carve_sigma_ao(Arena &ar, const Dims &d, int64_t nao, int mode) {
  SigmaAoBufs b{};
  const int64_t M = d.M;
  b.Xmo = ar.take<double>(M * d.n);
  if (fp64_mode(mode)) {
    b.Xs = ar.take<double>(M * d.n);
    b.Go = ar.take<double>(M * M);
    b.Gv = ar.take<double>(M * M);
    b.Zt = ar.take<double>(M * M);
    b.U = ar.take<double>(M * d.naux);
    b.R = ar.take<double>(M * nao);
    return b;
  }
  const int64_t naop = round_up(nao, 128);
  for (bf16 **q : {&b.D_hi, &b.D_lo, &b.U_hi, &b.U_lo}) *q = ar.take<bf16>(d.Mp * d.Ap);
  for (bf16 **q : {&b.W_hi, &b.W_lo}) *q = ar.take<bf16>(d.Ap * d.Ap);
  for (bf16 **q : {&b.Yo_hi, &b.Yo_lo}) *q = ar.take<bf16>(d.Mp * d.Ko);
  for (bf16 **q : {&b.Yv_hi, &b.Yv_lo}) *q = ar.take<bf16>(d.Mp * d.Kv);
  for (bf16 **q : {&b.Hl_hi, &b.Hl_lo, &b.Hg_hi, &b.Hg_lo}) *q = ar.take<bf16>(d.Mp * d.Mp);
  for (bf16 **q : {&b.XaT_hi, &b.XaT_lo, &b.RT_hi, &b.RT_lo}) *q = ar.take<bf16>(naop * d.Mp);
  b.Zf = ar.take<float>(d.Mp * d.Mp);
  return b;
}

size_t mbpt_sigma_ao_workspace_bytes(int64_t M, int64_t nao, int64_t norb, int64_t nocc,
                                     int64_t naux, int mode) {
  Dims d(M, norb, nocc, naux);
  if (!d.ok() || nao < 1 || !valid_mode(mode)) return SIZE_MAX;
  Arena ar;
  ar.counting = true;
  carve_sigma_ao(ar, d, nao, mode);
  return ar.used + 4096;
}

// Sigma^<(tau) = X_ao^T (G_occ o Zt) X_ao and Sigma^>(tau) = -X_ao^T (G_virt o
// Zt) X_ao per time point (GW/imaginary_time.py:403-533): the occupied/virtual
// split needs the MO collocation, the outer indices stay AO. FP64 modes:
// DGEMMs (or their int8 emulation) and Hadamard passes. Mixed: the engine's
// split products, as the self-energy sweep's: U = D W(tau), then one tile pass
// of G_occ, G_virt and Zt = U D^T whose epilogue forms H< = G_occ o Zt and
// H> = G_virt o Zt (upper tiles, mirrored), R^T = X_ao^T H (H symmetric), and
// X_ao^T R straight into the FP64 output by the symmetric FP64 epilogue.
int mbpt_sigma_ao(const double *X_ao, int64_t M, int64_t nao, const double *mo_coeff,
                  int64_t norb, int64_t nocc, const double *eps, double mu, const double *D,
                  int64_t naux, const double *Wt, const double *tau_host, int ntau, int mode,
                  double *out, void *ws, size_t ws_bytes, int *err, void *stream) {
  Dims d(M, norb, nocc, naux);
  if (!d.ok() || nao < 1 || ntau < 1) return MBPT_ERR_SHAPE;
  if (!valid_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  SigmaAoBufs b = carve_sigma_ao(ar, d, nao, mode);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  const int64_t nv = norb - nocc, a2 = naux * naux, o2 = nao * nao;
  if (!gemm_f64(h, false, false, M, norb, nao, 1.0, X_ao, nao, mo_coeff, norb, 0.0, b.Xmo,
                norb))
    return MBPT_ERR_CUDA;
  if (fp64_mode(mode)) {
    double *Xo_s = b.Xs, *Xv_s = b.Xs + M * nocc;
    for (int k = 0; k < ntau; ++k) {
      launch_scaled_branches(b.Xmo, M, norb, nocc, eps, mu, tau_host[k], 1.0, Xo_s, Xv_s, st);
      if (!gemm_mode(mode, h, false, true, M, M, nocc, 1.0, Xo_s, nocc, b.Xmo, norb, 0.0, b.Go,
                     M) ||
          !gemm_mode(mode, h, false, true, M, M, nv, 1.0, Xv_s, nv, b.Xmo + nocc, norb, 0.0,
                     b.Gv, M) ||
          !gemm_mode(mode, h, false, false, M, naux, naux, 1.0, D, naux, Wt + k * a2, naux,
                     0.0, b.U, naux) ||
          !gemm_mode(mode, h, false, true, M, M, naux, 1.0, b.U, naux, D, naux, 0.0, b.Zt, M,
                     true))
        return MBPT_ERR_CUDA;
      launch_hadamard(b.Go, b.Zt, M * M, st);
      launch_hadamard(b.Gv, b.Zt, M * M, st);
      if (!gemm_mode(mode, h, false, false, M, nao, M, 1.0, b.Go, M, X_ao, nao, 0.0, b.R,
                     nao) ||
          !gemm_mode(mode, h, true, false, nao, nao, M, 1.0, X_ao, nao, b.R, nao, 0.0,
                     out + k * o2, nao, true) ||
          !gemm_mode(mode, h, false, false, M, nao, M, 1.0, b.Gv, M, X_ao, nao, 0.0, b.R,
                     nao) ||
          !gemm_mode(mode, h, true, false, nao, nao, M, -1.0, X_ao, nao, b.R, nao, 0.0,
                     out + (ntau + k) * o2, nao, true))
        return MBPT_ERR_CUDA;
    }
    return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
  }
  const int64_t naop = round_up(nao, 128);
  launch_split_pad<double>(D, M, naux, naux, 1.f, b.D_hi, b.D_lo, d.Ap, d.Mp, d.Ap, false, st);
  launch_split_pad<double>(X_ao, M, nao, nao, 1.f, b.XaT_hi, b.XaT_lo, d.Mp, d.Mp, naop, true,
                           st);
  SplitMat Dm{b.D_hi, b.D_lo, d.Mp, d.Ap, d.Ap}, Wm{b.W_hi, b.W_lo, d.Ap, d.Ap, d.Ap};
  SplitMat Um{b.U_hi, b.U_lo, d.Mp, d.Ap, d.Ap};
  SplitMat Yo{b.Yo_hi, b.Yo_lo, d.Mp, d.Ko, d.Ko}, Yv{b.Yv_hi, b.Yv_lo, d.Mp, d.Kv, d.Kv};
  SplitMat Hl{b.Hl_hi, b.Hl_lo, d.Mp, d.Mp, d.Mp}, Hg{b.Hg_hi, b.Hg_lo, d.Mp, d.Mp, d.Mp};
  SplitMat XaT{b.XaT_hi, b.XaT_lo, naop, d.Mp, d.Mp}, RT{b.RT_hi, b.RT_lo, naop, d.Mp, d.Mp};
  for (int k = 0; k < ntau; ++k) {
    launch_prep_branches(b.Xmo, M, norb, nocc, eps, mu, tau_host[k], b.Yo_hi, b.Yo_lo, d.Ko,
                         b.Yv_hi, b.Yv_lo, d.Kv, d.Mp, st);
    launch_split_pad<double>(Wt + k * a2, naux, naux, naux, 1.f, b.W_hi, b.W_lo, d.Ap, d.Ap,
                             d.Ap, false, st);
    umma::EpiArgs e;
    e.out0_hi = b.U_hi;
    e.out0_lo = b.U_lo;
    e.ld_out = d.Ap;
    int rc = gemm_split(umma::EPI_SPLIT, 1, &Dm, &Wm, d.Mp, d.Ap, e, err, st);
    if (rc) return rc;
    // Zt = U D^T whole in FP32 (upper pair tiles, mirrored), then the G pass
    // H< = G_occ o Zt, H> = G_virt o Zt, as in the diagonal sweep
    e = umma::EpiArgs();
    e.outf = b.Zf;
    e.ld_outf = d.Mp;
    e.alpha = 1.f;
    rc = gemm_split(umma::EPI_F32, 1, &Um, &Dm, d.Mp, d.Mp, e, err, st, umma::BAND_UPPER);
    if (rc) return rc;
    e = umma::EpiArgs();
    e.out0_hi = b.Hl_hi;
    e.out0_lo = b.Hl_lo;
    e.out1_hi = b.Hg_hi;
    e.out1_lo = b.Hg_lo;
    e.ld_out = d.Mp;
    e.zt = b.Zf;
    e.ld_zt = d.Mp;
    SplitMat A2g[2] = {Yo, Yv};
    rc = gemm_split(umma::EPI_SIGMA_HZ, 2, A2g, A2g, d.Mp, d.Mp, e, err, st, umma::BAND_UPPER);
    if (rc) return rc;
    const SplitMat *H[2] = {&Hl, &Hg};
    for (int br = 0; br < 2; ++br) {
      e = umma::EpiArgs();
      e.out0_hi = b.RT_hi;
      e.out0_lo = b.RT_lo;
      e.ld_out = d.Mp;
      rc = gemm_split(umma::EPI_SPLIT, 1, &XaT, H[br], naop, d.Mp, e, err, st);
      if (rc) return rc;
      e = umma::EpiArgs();
      e.outd = out + (br * static_cast<int64_t>(ntau) + k) * o2;
      e.ld_outd = nao;
      e.nd = static_cast<int>(nao);
      e.shift = 0.0;
      e.alpha = br == 0 ? 1.f : -1.f;
      rc = gemm_split(umma::EPI_F64_SYM, 1, &XaT, &RT, naop, naop, e, err, st,
                      umma::BAND_UPPER);
      if (rc) return rc;
    }
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t mbpt_three_index_slices_workspace_bytes(int64_t M, int64_t norb) {
  return sizeof(double) * static_cast<size_t>(M) * norb + 2048;
}

int mbpt_three_index_slices(const double *X, int64_t M, int64_t norb, const double *D,
                            int64_t naux, const int64_t *states_host, int nstates, double *B,
                            void *ws, size_t ws_bytes, void *stream) {
  if (M < 1 || norb < 1 || naux < 1 || nstates < 1) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  double *T = ar.take<double>(M * norb);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  for (int s = 0; s < nstates; ++s) {
    const int64_t p = states_host[s];
    if (p < 0 || p >= norb) return MBPT_ERR_SHAPE;
    // B_p = D^T (x_p o X): LinearResponse/space_time.py:804-815
    launch_row_scaled_copy(X, M, norb, p, T, st);
    if (!gemm_f64(h, true, false, naux, norb, M, 1.0, D, naux, T, norb, 0.0,
                  B + static_cast<int64_t>(s) * naux * norb, norb))
      return MBPT_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// The explicit particle-hole response chi0 = s (C f) C^T. FP64: columns of C
// in chunks of kChi0AuxChunk, each chunk scaled into the workspace and folded
// into the lower triangle by row-panel DGEMMs, the other triangle mirrored.
// Mixed: C f and C as zero-padded BF16 pairs, one split product over the
// whole K on the engine's upper 128 x 256 tiles, stored as FP64 and mirrored
// by its epilogue.
constexpr int64_t kChi0AuxChunk = 4096;
constexpr int64_t kChi0AuxPanel = 1024;

size_t mbpt_chi0_aux_workspace_bytes(int64_t naux, int64_t nov, int mode) {
  if (naux < 1 || nov < 1) return 0;
  if (mode == MBPT_MODE_MIXED)
    return 4 * sizeof(bf16) * static_cast<size_t>(round_up(naux, 128)) * round_up(nov, 64) +
           4096;
  return sizeof(double) * static_cast<size_t>(naux) * std::min(nov, kChi0AuxChunk) + 2048;
}

int mbpt_chi0_aux(const double *C, int64_t naux, int64_t nov, int64_t ldc, const double *f,
                  double spin_factor, int accumulate, int mode, double *chi0, void *ws,
                  size_t ws_bytes, int *err, void *stream) {
  if (naux < 1 || nov < 1 || ldc < nov || naux > INT32_MAX || ldc > INT32_MAX)
    return MBPT_ERR_SHAPE;
  if (!valid_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  if (mode == MBPT_MODE_MIXED) {
    // the epilogue stores, it does not add
    if (accumulate) return MBPT_ERR_UNSUPPORTED;
    const int64_t mp = round_up(naux, 128), kp = round_up(nov, 64);
    bf16 *a_hi = ar.take<bf16>(mp * kp), *a_lo = ar.take<bf16>(mp * kp);
    bf16 *b_hi = ar.take<bf16>(mp * kp), *b_lo = ar.take<bf16>(mp * kp);
    if (ar.overflow()) return MBPT_ERR_WORKSPACE;
    launch_split_pad_colscale(C, naux, nov, ldc, f, spin_factor, a_hi, a_lo, kp, mp, kp, st);
    launch_split_pad<double>(C, naux, nov, ldc, 1.f, b_hi, b_lo, kp, mp, kp, false, st);
    SplitMat A{a_hi, a_lo, mp, kp, kp, false};
    SplitMat B{b_hi, b_lo, mp, kp, kp, false};
    umma::EpiArgs e;
    e.outd = chi0;
    e.ld_outd = naux;
    e.nd = static_cast<int>(naux);
    e.shift = 0.0;
    e.alpha = 1.f;
    const int rc = gemm_split(umma::EPI_F64_SYM, 1, &A, &B, mp, mp, e, err, st,
                              umma::BAND_UPPER);
    if (rc) return rc;
    return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
  }
  const int64_t chunk = std::min(nov, kChi0AuxChunk);
  double *T = ar.take<double>(naux * chunk);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  for (int64_t j0 = 0; j0 < nov; j0 += chunk) {
    const int64_t nc = std::min(chunk, nov - j0);
    launch_cols_scaled_copy(C, ldc, j0, f, spin_factor, naux, nc, T, st);
    const double beta = (j0 == 0 && !accumulate) ? 0.0 : 1.0;
    // the row-major lower triangle in row panels of kChi0AuxPanel: rows
    // [q0, q1) against columns [0, q1), one DGEMM each (the diagonal block
    // whole), the upper triangle mirrored once at the end
    for (int64_t q0 = 0; q0 < naux; q0 += kChi0AuxPanel) {
      const int64_t q1 = std::min(naux, q0 + kChi0AuxPanel);
      if (!dgemm_rm(h, false, true, q1 - q0, q1, nc, 1.0, T + q0 * nc, nc, C + j0, ldc, beta,
                    chi0 + q0 * naux, naux))
        return MBPT_ERR_CUDA;
    }
  }
  launch_mirror_lower_to_upper(chi0, naux, st);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// (1 - chi0) y = b from the Dyson step's Cholesky factor (column-major lower
// L, as mbpt_dyson leaves it with want_w = 0): two triangular solves on the
// nrhs right-hand sides of b (column-major n x nrhs), in place.
int mbpt_chol_solve(const double *L, int64_t n, double *b, int nrhs, void *stream) {
  if (n < 1 || nrhs < 1 || n > INT32_MAX) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  cublasHandle_t h = handles(st).blas;
  const double one = 1.0;
  const int ni = static_cast<int>(n);
  for (cublasOperation_t op : {CUBLAS_OP_N, CUBLAS_OP_T})
    if (cublasDtrsm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, op, CUBLAS_DIAG_NON_UNIT, ni,
                    nrhs, &one, L, ni, b, ni) != CUBLAS_STATUS_SUCCESS)
      return MBPT_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

struct ContractionBufs {
  double *Y = nullptr;                                        // fp64
  bf16 *w_hi = nullptr, *w_lo = nullptr, *b_hi = nullptr, *b_lo = nullptr;  // mixed
  float *y = nullptr;
  int64_t mp = 0, np = 0, kp = 0;
};

ContractionBufs carve_contraction(Arena &ar, int64_t naux, int64_t ncols, int mode) {
  ContractionBufs b;
  if (fp64_mode(mode)) {
    b.Y = ar.take<double>(naux * ncols);
    return b;
  }
  b.mp = round_up(naux, 128);
  b.np = round_up(ncols, 128);
  b.kp = round_up(naux, 64);
  b.w_hi = ar.take<bf16>(b.mp * b.kp);
  b.w_lo = ar.take<bf16>(b.mp * b.kp);
  b.b_hi = ar.take<bf16>(b.np * b.kp);
  b.b_lo = ar.take<bf16>(b.np * b.kp);
  b.y = ar.take<float>(b.mp * b.np);
  return b;
}

size_t mbpt_screening_contraction_workspace_bytes(int64_t naux, int64_t ncols, int mode) {
  Arena ar;
  ar.counting = true;
  carve_contraction(ar, naux, ncols, mode);
  return ar.used + 8192;
}

int mbpt_screening_contraction(const double *w_minus_i, int nfreq, int64_t naux,
                               const double *B, int64_t ncols, int mode, double *wc, void *ws,
                               size_t ws_bytes, int *err, void *stream) {
  if (nfreq < 1 || naux < 1 || ncols < 1) return MBPT_ERR_SHAPE;
  if (!valid_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  ContractionBufs c = carve_contraction(ar, naux, ncols, mode);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  if (cudaMemsetAsync(wc, 0, sizeof(double) * nfreq * ncols, st) != cudaSuccess)
    return MBPT_ERR_CUDA;
  if (mode == MBPT_MODE_MIXED) {
    // Y_k = (W - I)_k B as one split-BF16 product per frequency (FP32 out):
    // A = (W - I)_k (naux x naux), the second operand B^T (ncols x naux),
    // split once; then the column dots against B in FP64
    launch_split_pad<double>(B, naux, ncols, ncols, 1.f, c.b_hi, c.b_lo, c.kp, c.kp, c.np,
                             true, st);
    SplitMat Bm{c.b_hi, c.b_lo, c.np, c.kp, c.kp};
    for (int k = 0; k < nfreq; ++k) {
      launch_split_pad<double>(w_minus_i + k * naux * naux, naux, naux, naux, 1.f, c.w_hi,
                               c.w_lo, c.kp, c.mp, c.kp, false, st);
      SplitMat Am{c.w_hi, c.w_lo, c.mp, c.kp, c.kp};
      umma::EpiArgs e;
      e.outf = c.y;
      e.ld_outf = c.np;
      e.alpha = 1.f;
      int rc = gemm_split(umma::EPI_F32, 1, &Am, &Bm, c.mp, c.np, e, err, st);
      if (rc) return rc;
      launch_rowdot_f32(c.y, c.np, B, ncols, naux, ncols, wc + k * ncols, st);
    }
    return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
  }
  double *Y = c.Y;
  cublasHandle_t h = handles(st).blas;
  for (int k = 0; k < nfreq; ++k) {
    // wc[k, c] = B[:, c]^T (W - I)_k B[:, c]: GW/contour_deformation.py:229-237, 273-290
    if (!gemm_mode(mode, h, false, false, naux, ncols, naux, 1.0, w_minus_i + k * naux * naux,
                   naux, B, ncols, 0.0, Y, ncols))
      return MBPT_ERR_CUDA;
    launch_rowdot(Y, ncols, B, ncols, naux, ncols, 1.0, wc + k * ncols, st);
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t mbpt_cd_integral_backward_workspace_bytes(int64_t naux, int64_t norb) {
  return 2 * sizeof(double) * static_cast<size_t>(naux) * norb + 2048;
}

int mbpt_cd_integral_backward(const double *w_minus_i, int nfreq, int64_t naux, const double *B,
                              int64_t norb, const double *wc_bar, double *B_bar, double *W_bar,
                              void *ws, size_t ws_bytes, void *stream) {
  if (nfreq < 1 || naux < 1 || norb < 1) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  double *Y = ar.take<double>(naux * norb), *T = ar.take<double>(naux * norb);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  for (int k = 0; k < nfreq; ++k) {
    // wc[k, q] = b_q^T (W - I)_k b_q: B_bar += 2 ((W - I)_k B) diag(wc_bar[k]),
    // W_bar_k = B diag(wc_bar[k]) B^T (gradients/gwbse/qp_space_time.py:328-350)
    const double *v = wc_bar + k * norb;
    if (!gemm_f64(h, false, false, naux, norb, naux, 1.0, w_minus_i + k * naux * naux, naux, B,
                  norb, 0.0, Y, norb))
      return MBPT_ERR_CUDA;
    launch_col_scale(Y, v, naux, norb, 2.0, B_bar, true, st);
    launch_col_scale(B, v, naux, norb, 1.0, T, false, st);
    if (!gemm_f64(h, false, true, naux, naux, norb, 1.0, T, norb, B, norb, 0.0,
                  W_bar + k * naux * naux, naux))
      return MBPT_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t mbpt_three_index_slice_backward_workspace_bytes(int64_t M, int64_t norb, int64_t naux) {
  return sizeof(double) * static_cast<size_t>(M) * (norb > naux ? norb : naux) + 2048;
}

int mbpt_three_index_slice_backward(const double *X, int64_t M, int64_t norb, const double *D,
                                    int64_t naux, int64_t p, const double *B_bar, double *X_bar,
                                    double *D_bar, void *ws, size_t ws_bytes, void *stream) {
  if (M < 1 || norb < 1 || naux < 1 || p < 0 || p >= norb) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  Arena ar = arena(ws, ws_bytes);
  double *G = ar.take<double>(M * (norb > naux ? norb : naux));
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  cublasHandle_t h = handles(st).blas;
  // B_p = D^T diag(x_p) X (LinearResponse/space_time.py:804-815), its reverse
  // gradients/rpa/space_time_adjoint.py:593-624: G = D B_bar,
  // X_bar += diag(x_p) G, X_bar[:, p] += rowsum(G o X), D_bar += diag(x_p) X B_bar^T
  if (!gemm_f64(h, false, false, M, norb, naux, 1.0, D, naux, B_bar, norb, 0.0, G, norb))
    return MBPT_ERR_CUDA;
  launch_row_dot_into_col(G, X, M, norb, X_bar, norb, p, st);
  launch_row_scale_acc(X, norb, p, G, M, norb, X_bar, st);
  if (!gemm_f64(h, false, true, M, naux, norb, 1.0, X, norb, B_bar, norb, 0.0, G, naux))
    return MBPT_ERR_CUDA;
  launch_row_scale_acc(X, norb, p, G, M, naux, D_bar, st);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t mbpt_sigma_backward_workspace_bytes(int64_t M, int64_t norb, int64_t nocc,
                                           int64_t naux, int nstates) {
  Dims d(M, norb, nocc, naux);
  Arena ar;
  ar.counting = true;
  carve_sigma_back(ar, d, nstates > 0 ? nstates : 1);
  return ar.used + 2048;
}

int mbpt_sigma_backward(const double *X, int64_t M, int64_t norb, int64_t nocc,
                        const double *eps, double mu, const double *D, int64_t naux,
                        const double *tau, int ntau, const double *Wt, const int64_t *states,
                        int nstates, const double *sl_bar, const double *sg_bar, int mode,
                        double *eps_bar, double *X_bar, double *D_bar, double *Wt_bar,
                        void *ws, size_t ws_bytes, int *err, void *stream) {
  (void)err;
  Dims d(M, norb, nocc, naux);
  if (!d.ok() || ntau < 1 || nstates < 1) return MBPT_ERR_SHAPE;
  if (!fp64_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  Arena ar = arena(ws, ws_bytes);
  return sigma_back_run(X, d, eps, mu, D, tau, ntau, Wt, states, nstates, sl_bar, sg_bar,
                        eps_bar, X_bar, D_bar, Wt_bar, ar, S(stream), mode);
}

size_t mbpt_dyson_backward_workspace_bytes(int64_t naux) {
  return sizeof(double) * static_cast<size_t>(naux) * naux + 2048;
}

int mbpt_dyson_backward(const double *w_minus_i, double *wbar, int64_t naux, int nfreq,
                        int mode, void *ws, size_t ws_bytes, void *stream) {
  if (naux < 1 || nfreq < 1) return MBPT_ERR_SHAPE;
  if (!fp64_mode(mode)) return MBPT_ERR_UNSUPPORTED;
  Arena ar = arena(ws, ws_bytes);
  return dyson_back_run(w_minus_i, wbar, naux, nfreq, ar, S(stream), mode);
}

int mbpt_energy_adjoint_seed(double *wmi, int64_t naux, int nfreq, const double *ow_dev,
                             void *stream) {
  if (naux < 1 || nfreq < 1) return MBPT_ERR_SHAPE;
  launch_chi0_bar_seed(wmi, naux, nfreq, ow_dev, S(stream));
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t mbpt_dgemm_ozaki_workspace_bytes(int64_t m, int64_t n, int64_t k, int slices) {
  if (!gemm_extents_ok(m, n, k) || (slices != 7 && slices != 8)) return SIZE_MAX;
  return ozaki_gemm_scratch_bytes(m, n, k, slices);
}

int mbpt_dgemm_ozaki(int ta, int tb, int64_t m, int64_t n, int64_t k, double alpha,
                     const double *A, int64_t lda, const double *B, int64_t ldb, double beta,
                     double *C, int64_t ldc, int slices, void *ws, size_t ws_bytes, int *err,
                     void *stream) {
  if (!gemm_extents_ok(m, n, k) || ldc < n || lda < (ta ? m : k) || ldb < (tb ? k : n))
    return MBPT_ERR_SHAPE;
  return ozaki_dgemm(ta != 0, tb != 0, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, slices,
                     ws, ws_bytes, err, S(stream));
}

size_t mbpt_gemm_split_tf32_workspace_bytes(int64_t m, int64_t n, int64_t k) {
  if (!gemm_extents_ok(m, n, k)) return SIZE_MAX;
  const int64_t mp = round_up(m, 128), np = round_up(n, 128), kp = round_up(k, 32);
  Arena ar;
  ar.counting = true;
  ar.take<float>(mp * kp);
  ar.take<float>(mp * kp);
  ar.take<float>(np * kp);
  ar.take<float>(np * kp);
  ar.take<float>(mp * np);
  return ar.used + 8192;
}

int mbpt_gemm_split_tf32(const double *A, const double *B, int64_t m, int64_t n, int64_t k,
                         double alpha, float *C, int64_t ldc, void *ws, size_t ws_bytes,
                         int *err, void *stream) {
  if (!gemm_extents_ok(m, n, k) || ldc < n) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  const int64_t mp = round_up(m, 128), np = round_up(n, 128), kp = round_up(k, 32);
  Arena ar = arena(ws, ws_bytes);
  float *a_hi = ar.take<float>(mp * kp), *a_lo = ar.take<float>(mp * kp);
  float *b_hi = ar.take<float>(np * kp), *b_lo = ar.take<float>(np * kp);
  float *c = ar.take<float>(mp * np);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  launch_split_pad_tf32(A, m, k, k, a_hi, a_lo, kp, mp, kp, st);
  launch_split_pad_tf32(B, n, k, k, b_hi, b_lo, kp, np, kp, st);
  SplitMat Am{a_hi, a_lo, mp, kp, kp, true}, Bm{b_hi, b_lo, np, kp, kp, true};
  umma::EpiArgs e;
  e.outf = c;
  e.ld_outf = np;
  e.alpha = static_cast<float>(alpha);
  int rc = gemm_split(umma::EPI_F32, 1, &Am, &Bm, mp, np, e, err, st);
  if (rc) return rc;
  cudaMemcpy2DAsync(C, sizeof(float) * ldc, c, sizeof(float) * np, sizeof(float) * n, m,
                    cudaMemcpyDeviceToDevice, st);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

size_t mbpt_gemm_split_workspace_bytes(int64_t m, int64_t n, int64_t k) {
  if (!gemm_extents_ok(m, n, k)) return SIZE_MAX;
  const int64_t mp = round_up(m, 128), np = round_up(n, 128), kp = round_up(k, 64);
  Arena ar;
  ar.counting = true;
  ar.take<bf16>(2 * mp * kp);
  ar.take<bf16>(2 * np * kp);
  ar.take<float>(mp * np);
  return ar.used + 8192;
}

int mbpt_gemm_split(const double *A, const double *B, int64_t m, int64_t n, int64_t k,
                    double alpha, float *C, int64_t ldc, void *ws, size_t ws_bytes, int *err,
                    void *stream) {
  if (!gemm_extents_ok(m, n, k) || ldc < n) return MBPT_ERR_SHAPE;
  cudaStream_t st = S(stream);
  const int64_t mp = round_up(m, 128), np = round_up(n, 128), kp = round_up(k, 64);
  Arena ar = arena(ws, ws_bytes);
  bf16 *a_hi = ar.take<bf16>(mp * kp), *a_lo = ar.take<bf16>(mp * kp);
  bf16 *b_hi = ar.take<bf16>(np * kp), *b_lo = ar.take<bf16>(np * kp);
  float *c = ar.take<float>(mp * np);
  if (ar.overflow()) return MBPT_ERR_WORKSPACE;
  launch_split_pad<double>(A, m, k, k, 1.f, a_hi, a_lo, kp, mp, kp, false, st);
  launch_split_pad<double>(B, n, k, k, 1.f, b_hi, b_lo, kp, np, kp, false, st);
  SplitMat Am{a_hi, a_lo, mp, kp, kp}, Bm{b_hi, b_lo, np, kp, kp};
  umma::EpiArgs e;
  e.outf = c;
  e.ld_outf = np;
  e.alpha = static_cast<float>(alpha);
  int rc = gemm_split(umma::EPI_F32, 1, &Am, &Bm, mp, np, e, err, st);
  if (rc) return rc;
  cudaMemcpy2DAsync(C, sizeof(float) * ldc, c, sizeof(float) * np, sizeof(float) * n, m,
                    cudaMemcpyDeviceToDevice, st);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

}  // extern "C"
