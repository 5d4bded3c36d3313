// Internal (C++) interface between the route orchestration and the kernels.
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include "umma_gemm.cuh"

namespace mbpt {

// A split operand x = hi + lo: rows x cols (cols = K, contiguous), leading
// dimension ld, elements BF16 (tf32 false) or TF32-rounded FP32 words.
struct SplitMat {
  const void *hi = nullptr, *lo = nullptr;
  int64_t rows = 0, cols = 0, ld = 0;
  bool tf32 = false;
};

// C (m_rows x n_rows tile grid, both multiples of 128) from nacc problems
// A[j] B[j]^T with the fused epilogue `epi`. band: umma::Band flags of
// triangular operands (the TF32 single-product FP32 store only).
int gemm_split(int epi, int nacc, const SplitMat *A, const SplitMat *B, int64_t m_rows,
               int64_t n_rows, const umma::EpiArgs &e, int *err, cudaStream_t st,
               int band = 0);

// One product of a grouped launch: an m_rows x n_rows output block (multiples
// of 128) from the A rows [a_row0, +m_rows) and B rows [b_row0, +n_rows), K
// elements from a_k0 / b_k0 (multiples of 32), output origins at element
// offsets p_off / t_off of the epilogue's arrays.
struct GemmGroup {
  int64_t m_rows, n_rows, k;
  int64_t a_row0, a_k0, b_row0, b_k0;
  int64_t p_off, t_off;
};
// Independent single-accumulator TF32 products of the same A and B arrays in
// as few launches as possible (up to 32 per launch); EPI_TF32_PAIR only.
int gemm_split_grouped(int epi, const SplitMat &A, const SplitMat &B, const GemmGroup *groups,
                       int ngroups, const umma::EpiArgs &e, int *err, cudaStream_t st,
                       int band = 0);

// The engine's bounded barrier wait on a barrier that is (arrive = 1) or is
// never (arrive = 0) completed, giving up after limit_us microseconds.
int wait_selftest(int arrive, int64_t limit_us, int *err, cudaStream_t st);

// Per-epilogue totals of the engine's launch times (enable = 1 starts
// recording; a call with non-null outputs drains, returns and resets them).
int gemm_timing(int enable, double *total_ms, long long *launches);
// Records the calling thread's next engine launches under category `tag`
// instead of their epilogue kind (-1: back to the epilogue kind).
void timing_tag(int tag);
constexpr int kTimingDyson = 7;  // TF32 products of the Dyson step's inverse

// cuTensorMapEncodeTiled through the runtime's driver entry point (null when
// the driver lacks it), and a kernel's dynamic shared-memory opt-in, once per
// device (one bit per device in `done`).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn();
bool allow_smem(const void *kern, int bytes, std::atomic<uint64_t> &done);

// ---- Ozaki-scheme FP64 updates of the batched Cholesky (ozaki.cu) ----
// Largest K (matrix size) of the 8-bit digit updates (slices = 6): 6 127^2 K < 2^31.
constexpr int64_t kOzakiEightBitMaxK = 22016;
// Bytes of the int8 digit planes of nmat n x n factors cut into `slices`.
size_t ozaki_planes_bytes(int64_t n, int nmat, int slices);
// scale[f][r] = 2^e_r >= sqrt(A_rr) of each matrix (column-major, ld n; of
// I - A with one_minus); the running row norms rownorm (nmat x n) start at zero.
int ozaki_chol_scales(const double *A, int64_t n, int nmat, double *scale, double *rownorm,
                      bool one_minus, cudaStream_t st);
// Cut block column [j0, j0 + nb) of every factor (rows j0..n-1) into digit
// planes, adding its squares to the rows' running norms.
int ozaki_chol_slice(const double *A, int64_t n, int nmat, int64_t j0, int nb,
                     const double *scale, int8_t *planes, int slices, double *rownorm,
                     cudaStream_t st);
// P -= L[j0:, :j0] L[j0:j0+nb, :j0]^T for every matrix from the digit planes
// (the diagonal entries from the exact FP64 running row norms, nmat x n).
int ozaki_chol_update(double *A, int64_t n, int nmat, int64_t j0, int nb, double *P,
                      const double *scale, const int8_t *planes, int slices, double *rowsq,
                      int *err, cudaStream_t st);
// C (m x n, row-major, ldc) = alpha op(A) op(B) + beta C in FP64 accuracy on
// the int8 tensor cores (Ozaki scheme, `slices` digits per operand, 7 or 8):
// op(A) = A (m x k, lda) or, with ta, A^T of a k x m A; op(B) = B (k x n,
// ldb) or, with tb, B^T of an n x k B. scratch: ozaki_gemm_scratch_bytes.
// Options of the epilogue (null: a plain product):
//   sym: the product is known to be symmetric (m == n): the tiles on and
//        above the diagonal are formed and mirrored, the others skipped;
//   h1 (and h2): C = (alpha op(A) op(B)) o h1 and C2 = (alpha op(A) op(B)) o h2,
//        element-wise, h1, h2 and C2 with C's leading dimension; needs beta
//        0 and k <= kOzakiKChunk (the product complete in one pass).
struct OzakiEpi {
  bool sym = false;
  const double *h1 = nullptr, *h2 = nullptr;
  double *c2 = nullptr;
};
constexpr int64_t kOzakiKChunk = 32768;
size_t ozaki_gemm_scratch_bytes(int64_t m, int64_t n, int64_t k, int slices);
int ozaki_dgemm(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                const double *A, int64_t lda, const double *B, int64_t ldb, double beta,
                double *C, int64_t ldc, int slices, void *scratch, size_t scratch_bytes,
                int *err, cudaStream_t st, const OzakiEpi *epi = nullptr);

// Bump allocator over a caller's workspace (1024-byte aligned slices).
struct Arena {
  uint8_t *base = nullptr;
  size_t size = 0, used = 0;
  bool counting = false;  // size-query mode: hand out nothing, count bytes
  template <typename T>
  T *take(size_t count) {
    size_t off = (used + 1023) & ~static_cast<size_t>(1023);
    size_t bytes = count * sizeof(T);
    used = off + bytes;
    if (counting) return nullptr;
    if (used > size) return nullptr;
    return reinterpret_cast<T *>(base + off);
  }
  bool overflow() const { return !counting && used > size; }
};

// ---- elementwise / bandwidth kernels (kernels.cu) ----
template <typename T>
void launch_split_pad(const T *src, int64_t rows, int64_t cols, int64_t ld_src, float scale,
                      bf16 *hi, bf16 *lo, int64_t ld_dst, int64_t rows_p, int64_t cols_p,
                      bool transpose, cudaStream_t st);
void launch_prep_branches(const double *X, int64_t M, int64_t n, int64_t nocc,
                          const double *eps, double mu, double tau, bf16 *o_hi, bf16 *o_lo,
                          int64_t ld_o, bf16 *v_hi, bf16 *v_lo, int64_t ld_v, int64_t Mp,
                          cudaStream_t st);
void launch_prep_branches_tf32(const double *X, int64_t M, int64_t n, int64_t nocc,
                               const double *eps, double mu, double tau, float *o_hi,
                               float *o_lo, int64_t ld_o, float *v_hi, float *v_lo,
                               int64_t ld_v, int64_t Mp, cudaStream_t st);
void launch_split_pad_colscale(const double *src, int64_t rows, int64_t cols, int64_t ld_src,
                               const double *f, double s, bf16 *hi, bf16 *lo, int64_t ld_dst,
                               int64_t rows_p, int64_t cols_p, cudaStream_t st);
void launch_split_pad_tf32(const double *src, int64_t rows, int64_t cols, int64_t ld_src,
                           float *hi, float *lo, int64_t ld_dst, int64_t rows_p, int64_t cols_p,
                           cudaStream_t st);
void launch_scaled_branches(const double *X, int64_t M, int64_t n, int64_t nocc,
                            const double *eps, double mu, double tau, double power,
                            double *Xo_s, double *Xv_s, cudaStream_t st);
void launch_hadamard(double *a, const double *b, int64_t n, cudaStream_t st);
void launch_hadamard3(double *out, const double *a, const double *b, int64_t n, cudaStream_t st);
// out[j] = sum_k w[j,k] in[k] over a rows x cols block of each slice
template <typename Tin>
void launch_transform(const Tin *in, int64_t in_slice, int64_t ld_in, int64_t rows,
                      int64_t cols, const double *w_dev, int J, int K, double *out,
                      int64_t out_slice, int64_t ld_out, cudaStream_t st);
// out[j] += sum_k w[j,k] in[k] (FP64)
void launch_transform_acc(const double *in, int64_t in_slice, int64_t ld_in, int64_t rows,
                          int64_t cols, const double *w_dev, int J, int K, double *out,
                          int64_t out_slice, int64_t ld_out, cudaStream_t st);
// a <- I - a per n x n slice; with trace, trace[f] = tr a first
void launch_one_minus(double *a, int64_t n, int nmat, double *trace, cudaStream_t st);
void launch_trace(const double *a, int64_t n, int nmat, double *trace, cudaStream_t st);
void launch_logdet_diag(const double *L, int64_t n, int nmat, double *logdet,
                        cudaStream_t st);
void launch_symmetrize_minus_identity(double *a, int64_t n, int nmat, cudaStream_t st);
void launch_rowdot(const double *R, int64_t ld_r, const double *Xs, int64_t ld_x, int64_t M,
                   int64_t S, double sign, double *out, cudaStream_t st);
void launch_gather_cols_f32(const double *X, int64_t M, int64_t n, const int64_t *states,
                            int64_t S, float *xs, int64_t ld_xs, int64_t Mp, cudaStream_t st);
void launch_gather_cols_split_t(const double *X, int64_t M, int64_t n, const int64_t *states,
                                int64_t S, bf16 *hi, bf16 *lo, int64_t ld, int64_t Sp,
                                int64_t Mp, cudaStream_t st);
void launch_gather_cols_f64(const double *X, int64_t M, int64_t n, const int64_t *states,
                            int64_t S, double *xs, cudaStream_t st);
void launch_sigma_frequency(const double *branch, int ntau, int nstates, const double *C,
                            const double *S, int npade, double *sigma, cudaStream_t st);
void launch_energy_sum(const double *logdet, const double *trace, const double *w, int nfreq,
                       double *e_c, cudaStream_t st);

}  // namespace mbpt
