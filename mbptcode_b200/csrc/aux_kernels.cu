// Small FP64 kernels of the adjoint and of the Dyson step (its triangular
// inverse and the FP64 <-> TF32-pair conversions of its tensor-core products).
#include <cmath>

#include "internal.h"

namespace mbpt {
namespace {

inline int blocks(int64_t n) {
  int64_t b = (n + 255) / 256;
  return static_cast<int>(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

// a_f <- -(w_f / 2pi) a_f^T for each W - I slice: chi0_bar of the dRPA energy
// (W - I is symmetric here, the mirrored output of the Dyson step).
__global__ void chi0_bar_seed_kernel(double *a, int64_t n, const double *w) {
  double *m = a + static_cast<int64_t>(blockIdx.y) * n * n;
  const double s = -w[blockIdx.y] / (2.0 * 3.14159265358979323846);
  const int64_t total = n * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    m[i] *= s;
}

// out = (in + in^T) / 2
__global__ void sym_half_kernel(const double *in, double *out, int64_t n) {
  const int64_t total = n * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i % n;
    out[i] = 0.5 * (in[i] + in[c * n + r]);
  }
}

// X_bar[:, occ] += 2 GoX w, X_bar[:, virt] += 2 GvX u;
// eps_bar[i] += tau w_i sum_b X[b,i] GoX[b,i], eps_bar[a] -= tau u_a sum_b X[b,a] GvX[b,a]
__global__ void xbar_kernel(const double *GoX, const double *GvX, const double *X, int64_t M,
                            int64_t n, int64_t nocc, const double *eps, double mu, double tau,
                            double *X_bar, double *eps_bar) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * 32 + threadIdx.x;
  __shared__ double part[8][33];
  const int64_t nv = n - nocc;
  double s = 0.0;
  double f = 0.0;
  if (c < n) {
    const bool occ = c < nocc;
    f = occ ? exp((eps[c] - mu) * tau) : exp(-(eps[c] - mu) * tau);
    const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 256;
    const int64_t r1 = min(r0 + 256, M);
    for (int64_t r = r0 + threadIdx.y; r < r1; r += 8) {
      const double g = occ ? GoX[r * nocc + c] : GvX[r * nv + (c - nocc)];
      X_bar[r * n + c] += 2.0 * g * f;
      s += X[r * n + c] * g;
    }
  }
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && c < n) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x];
    const double sign = c < nocc ? 1.0 : -1.0;
    atomicAdd(eps_bar + c, sign * tau * f * t);
  }
}

// restore a symmetric matrix from its row-major lower triangle
__global__ void mirror_kernel(double *a, int64_t n) {
  const int64_t total = n * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i % n;
    if (r < c) a[i] = a[c * n + r];
  }
}

// log|det| and sign from an LU factor with 1-based pivots (column-major view)
__global__ void lu_logdet_kernel(const double *LU, const int *piv, int64_t n, double *logdet,
                                 int *sign) {
  __shared__ double part[256];
  __shared__ int neg[256];
  double s = 0.0;
  int ng = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double d = LU[i * n + i];
    s += log(fabs(d));
    if (d < 0.0) ng ^= 1;
    if (piv[i] != i + 1) ng ^= 1;
  }
  part[threadIdx.x] = s;
  neg[threadIdx.x] = ng;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      part[threadIdx.x] += part[threadIdx.x + w];
      neg[threadIdx.x] ^= neg[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *logdet = part[0];
    *sign = neg[0] ? -1 : 1;
  }
}

// diag[f * n + i] <-> a_f[i, i]
__global__ void diag_kernel(double *a, int64_t n, double *diag, bool save) {
  double *m = a + static_cast<int64_t>(blockIdx.y) * n * n;
  double *d = diag + static_cast<int64_t>(blockIdx.y) * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (save)
      d[i] = m[i * n + i];
    else
      m[i * n + i] = d[i];
  }
}

// T (ib x ib, column-major) = the lower triangle of the column-major block at
// A (leading dimension lda), zeros above the diagonal
__global__ void lower_copy_kernel(const double *A, int64_t lda, double *T, int ib) {
  const int64_t total = static_cast<int64_t>(ib) * ib;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = i / ib, r = i % ib;
    T[i] = r >= c ? A[c * lda + r] : 0.0;
  }
}

// zero the strict upper triangle of a column-major n x n matrix (the
// row-major strict lower triangle of the buffer)
__global__ void zero_strict_upper_cm_kernel(double *a, int64_t n) {
  const int64_t total = n * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = i / n, r = i % n;  // column-major (r, c) at c * n + r
    if (r < c) a[i] = 0.0;
  }
}

// Inverts the nb x nb diagonal blocks of a column-major lower-triangular
// matrix in place, one CTA per block: the block is staged row-major in shared
// memory and inverted row by row (forward substitution against the rows
// already inverted), so the block never leaves the SM until it is done.
// With c_hi set, the inverted blocks go out as TF32 pairs instead, in two
// layouts of the padded (ldp) pair arrays: rows of L^-1 (r_*) and columns of
// L^-1 as rows (c_*), zeros above the diagonal included; A keeps the factor.
// The row recursion's dot products are split over kDiagParts threads per
// column (partial sums combined by warp shuffles), and the block is stored
// with a padded row stride so the parts' reads fall in different banks.
constexpr int kDiagParts = 4;

__global__ void trtri_diag_blocks_kernel(double *A, int64_t n, int64_t lda, int nb, float *c_hi,
                                         float *c_lo, float *r_hi, float *r_lo, int64_t ldp) {
  extern __shared__ double s[];  // m x m row-major block (stride m + 1), then one row of L
  const int64_t off = static_cast<int64_t>(blockIdx.x) * nb;
  const int m = static_cast<int>(min(static_cast<int64_t>(nb), n - off));
  const int ls = m + 1;
  double *row = s + m * ls;
  for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
    const int r = idx / m, c = idx % m;
    s[r * ls + c] = r >= c ? A[(off + c) * lda + off + r] : 0.0;
  }
  __syncthreads();
  const int j = threadIdx.x / kDiagParts, part = threadIdx.x % kDiagParts;
  for (int i = 0; i < m; ++i) {
    for (int k = threadIdx.x; k <= i; k += blockDim.x) row[k] = s[i * ls + k];
    __syncthreads();
    const double inv = 1.0 / row[i];
    // row i of L^-1: (L^-1)_ij = -(sum_{j<=k<i} L_ik (L^-1)_kj) / L_ii
    double acc = 0.0;
    if (j < i)
      for (int k = j + part; k < i; k += kDiagParts) acc = fma(row[k], s[k * ls + j], acc);
#pragma unroll
    for (int d = 1; d < kDiagParts; d <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
    if (part == 0 && j <= i) s[i * ls + j] = j == i ? inv : -acc * inv;
    __syncthreads();
  }
  if (c_hi) {
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
      const int r = idx / m, c = idx % m;
      const double x = s[r * ls + c];
      const float h = to_tf32(static_cast<float>(x));
      const float l = to_tf32(static_cast<float>(x - static_cast<double>(h)));
      r_hi[(off + r) * ldp + off + c] = h;
      r_lo[(off + r) * ldp + off + c] = l;
      c_hi[(off + c) * ldp + off + r] = h;
      c_lo[(off + c) * ldp + off + r] = l;
    }
    return;
  }
  for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
    const int r = idx / m, c = idx % m;
    if (r >= c) A[(off + c) * lda + off + r] = s[r * ls + c];
  }
}

// dst (rows_p x k_p row-major TF32 hi/lo pairs, zero padded) of the logical
// rows x k FP64 matrix X(r, c) = src[r * rs + c * cs], through a 32 x 33
// shared tile so that the global reads run along whichever stride is 1.
// The pair is split from the FP64 value: hi = tf32(x), lo = tf32(x - hi).
__global__ void strided_to_tf32_kernel(const double *__restrict__ src, int64_t rows, int64_t k,
                                       int64_t rs, int64_t cs, float *hi, float *lo,
                                       int64_t rows_p, int64_t k_p) {
  __shared__ double tile[32][33];
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 32;
  const int64_t c0 = static_cast<int64_t>(blockIdx.x) * 32;
  const bool col_unit = cs == 1;
  for (int a = threadIdx.y; a < 32; a += blockDim.y) {
    const int64_t r = col_unit ? r0 + a : r0 + threadIdx.x;
    const int64_t c = col_unit ? c0 + threadIdx.x : c0 + a;
    const double v = (r < rows && c < k) ? src[r * rs + c * cs] : 0.0;
    if (col_unit)
      tile[a][threadIdx.x] = v;
    else
      tile[threadIdx.x][a] = v;
  }
  __syncthreads();
  for (int a = threadIdx.y; a < 32; a += blockDim.y) {
    const int64_t r = r0 + a, c = c0 + threadIdx.x;
    if (r < rows_p && c < k_p) {
      const double x = tile[a][threadIdx.x];
      const float h = to_tf32(static_cast<float>(x));
      hi[r * k_p + c] = h;
      lo[r * k_p + c] = to_tf32(static_cast<float>(x - static_cast<double>(h)));
    }
  }
}

__global__ void identity_kernel(double *a, int64_t n, double diag_shift, bool set) {
  const int64_t total = n * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i % n;
    if (set)
      a[i] = (r == c) ? 1.0 : 0.0;
    else if (r == c)
      a[i] += diag_shift;
  }
}

// ---------------------------------------------------------- self-energy adjoint
// Xs[r, s] = X[r, states[s]] scaled by the branch adjoints of one tau point:
// Xl = Xs diag(sl), Xg = Xs diag(sg) (MBPTcode gradients/rpa/space_time_adjoint.py:846-853,
// there as the weights c of the bra slice)
__global__ void sigma_back_gather_kernel(const double *__restrict__ X, int64_t M, int64_t n,
                                         const int64_t *__restrict__ states, int64_t S,
                                         const double *__restrict__ sl,
                                         const double *__restrict__ sg, double *Xs, double *Xl,
                                         double *Xg) {
  const int64_t total = M * S;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / S, c = i % S;
    const double x = X[r * n + states[c]];
    Xs[i] = x;
    Xl[i] = x * sl[c];
    Xg[i] = x * sg[c];
  }
}

// The elementwise reverse of Sigma^<_s = x_s^T (Go o Zt) x_s and
// Sigma^>_s = -x_s^T (Gv o Zt) x_s with Al = sum_s sl_s x_s x_s^T and
// Ag = sum_s sg_s x_s x_s^T, in place:
//   zt <- Zt_bar = go al - gv ag,  al <- Go_bar = zt al,  ag <- Gv_bar = -zt ag,
//   go <- L = go zt,               gv <- H = gv zt
__global__ void sigma_back_hadamard_kernel(double *go, double *gv, double *zt, double *al,
                                           double *ag, int64_t total) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double o = go[i], v = gv[i], z = zt[i], a = al[i], g = ag[i];
    zt[i] = o * a - v * g;
    al[i] = z * a;
    ag[i] = -z * g;
    go[i] = o * z;
    gv[i] = v * z;
  }
}

// X_bar[r, states[s]] += scale * T[r, s] (a state listed twice adds twice)
__global__ void scatter_cols_kernel(const double *__restrict__ T, int64_t M, int64_t S,
                                    const int64_t *__restrict__ states, double scale,
                                    double *X_bar, int64_t n) {
  const int64_t total = M * S;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / S, c = i % S;
    atomicAdd(X_bar + r * n + states[c], scale * T[i]);
  }
}

// ------------------------------------------------ batched blocked Cholesky
// One 128-column step of the left-looking Cholesky of a batch of column-major
// n x n matrices (the lower factor, as cuSOLVER's lower-fill potrf leaves it;
// the strict upper triangle is never written).
constexpr int kCholNb = 128;
constexpr int kCholStride = kCholNb + 1;  // odd: a column of s read by a warp is free of bank conflicts

// P_f (m x nbj, column-major, ld m) <- the block column A_f[j0:, j0:j0+nbj],
// or of I - A_f with one_minus (the factorised matrix is then I - A_f, whose
// entries are formed here, each read once)
__global__ void chol_copy_panel_kernel(const double *__restrict__ A, int64_t n, int64_t j0,
                                       int64_t m, int nbj, bool one_minus,
                                       double *__restrict__ P) {
  const double *a = A + static_cast<int64_t>(blockIdx.y) * n * n;
  double *p = P + static_cast<int64_t>(blockIdx.y) * m * nbj;
  const int64_t total = m * nbj;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = i / m, r = i % m;
    const double v = a[(j0 + c) * n + j0 + r];
    p[i] = one_minus ? (r == c ? 1.0 : 0.0) - v : v;
  }
}

// One CTA (512 threads) per matrix: the updated diagonal block (the top nbj
// rows of P_f, padded to 128 with the identity) is factorised and inverted in
// shared memory, blocked by 32-column sub-blocks so that the sequential part,
// one pivot after another, stays inside one warp:
//  * warp 0 factorises the 32 x 32 diagonal sub-block in registers (lane r
//    holds row r; each pivot's column is broadcast by shuffles, the chain per
//    column is one rsqrt and one FMA) and forms its inverse X_kk by forward
//    substitution column by column (lane c holds column c);
//  * all warps then form the rows below it, L_ik = A_ik X_kk^T, and apply the
//    rank-32 update of the trailing lower triangle in 4 x 4 register tiles;
//  * after the last sub-block the off-diagonal blocks of X = L^-1 follow by
//    block rows, X_ik = -X_ii sum_{k <= j < i} L_ij X_jk.
// The lower factor goes into A_f's diagonal block (lower triangle and
// diagonal only), X into Linv_f (column-major, ld kCholNb, zeros above the
// diagonal). The diagonal is sqrt(pivot), the scaling of the column below it
// rsqrt(pivot) (within an ulp of LAPACK's 1 / sqrt). A pivot that is not
// positive records info_f = its global column + 1 (the first one only), as
// potrf does; the factor of that matrix is then not meaningful.
// Shared memory: s (128 x kCholStride: L in the strict lower triangle, the
// off-diagonal blocks of X transposed in the upper one, X[r][c] at s[c][r]),
// the diagonal of L and of X, the four X_kk dense (kCholXStride rows), and
// the current panel transposed (pt, reused for the block products of the
// inverse).
constexpr int kCholSub = 32;
constexpr int kCholXStride = kCholSub + 1;
constexpr int kCholPtStride = kCholNb + 2;  // even: the 4 x 4 tiles read pairs
constexpr int kCholSmemDoubles = kCholNb * kCholStride + 2 * kCholNb +
                                 (kCholNb / kCholSub) * kCholSub * kCholXStride +
                                 kCholSub * kCholPtStride;

__global__ void __launch_bounds__(512) chol_diag_block_kernel(
    const double *__restrict__ P, int64_t m, int nbj, double *A, int64_t n, int64_t j0,
    double *__restrict__ Linv, int *info) {
  extern __shared__ __align__(16) double sm[];
  constexpr int ST = kCholStride, XS = kCholXStride, PT = kCholPtStride, NB = kCholNb;
  double *s = sm;
  double *diag = s + NB * ST;                 // L_cc
  double *xdiag = diag + NB;                  // X_cc = rsqrt(pivot)
  double *xd = xdiag + NB;                    // X_kk dense, [k][r][c]
  double *pt = xd + (NB / kCholSub) * kCholSub * XS;  // panel transposed, [m][i]
  double *tb = pt;                            // the inverse's block products, [k][r][c]
  __shared__ int bad;
  const int f = blockIdx.x, tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  const double *p = P + static_cast<int64_t>(f) * m * nbj;
  double *a = A + static_cast<int64_t>(f) * n * n;
  if (tid == 0) bad = -1;
  // the tile padded with the identity, zeros above the diagonal; eight
  // independent loads in flight per thread before any store
  for (int i0 = tid; i0 < NB * NB; i0 += 8 * blockDim.x) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * blockDim.x;
      const int c = i / NB, r = i % NB;
      v[u] = 0.0;
      if (i < NB * NB && r >= c)
        v[u] = (r < nbj && c < nbj) ? p[static_cast<int64_t>(c) * m + r] : (r == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < NB * NB) s[(i % NB) * ST + i / NB] = v[u];
    }
  }
  __syncthreads();
  for (int k = 0; k < NB / kCholSub; ++k) {
    const int b = k * kCholSub;
    double *xk = xd + k * kCholSub * XS;
    if (warp == 0) {
      double *row = s + (b + lane) * ST + b;
      double v[kCholSub];
#pragma unroll
      for (int j = 0; j < kCholSub; ++j) v[j] = row[j];
      // right-looking in registers: entries of a lane above the diagonal
      // are never read by another lane
#pragma unroll
      for (int c = 0; c < kCholSub; ++c) {
        const double d = __shfl_sync(0xffffffffu, v[c], c);
        const double rs = rsqrt(d);
        if (lane == 0) {
          xdiag[b + c] = rs;
          diag[b + c] = sqrt(d);
          if (!(d > 0.0) && bad < 0 && b + c < nbj) bad = b + c;
        }
        v[c] *= rs;
#pragma unroll
        for (int j = c + 1; j < kCholSub; ++j)
          v[j] = fma(-v[c], __shfl_sync(0xffffffffu, v[c], j), v[j]);
      }
#pragma unroll
      for (int j = 0; j < kCholSub; ++j)
        if (j < lane) row[j] = v[j];
      __syncwarp();
      // X_kk column `lane`: x_i = (e_lane - sum_{j < i} L_ij x_j) / L_ii,
      // the sums carried forward so that the chain per row is one FMA
      double x[kCholSub];
#pragma unroll
      for (int r = 0; r < kCholSub; ++r) x[r] = r == lane ? 1.0 : 0.0;
#pragma unroll
      for (int i = 0; i < kCholSub; ++i) {
        x[i] *= xdiag[b + i];
#pragma unroll
        for (int r = i + 1; r < kCholSub; ++r) x[r] = fma(-s[(b + r) * ST + b + i], x[i], x[r]);
      }
#pragma unroll
      for (int r = 0; r < kCholSub; ++r) xk[r * XS + lane] = x[r];
    }
    __syncthreads();
    if (b + kCholSub >= NB) break;
    // the rows below: L[i][b + j] = sum_q A[i][b + q] X_kk[j][q], two rows per warp pass
    for (int i0 = b + kCholSub + 2 * warp; i0 < NB; i0 += 2 * nwarps) {
      double *r0 = s + i0 * ST + b, *r1 = r0 + ST;
      double acc0 = 0.0, acc1 = 0.0;
#pragma unroll 8
      for (int q = 0; q < kCholSub; ++q) {
        const double x = xk[lane * XS + q];
        acc0 = fma(r0[q], x, acc0);
        acc1 = fma(r1[q], x, acc1);
      }
      __syncwarp();
      r0[lane] = acc0;
      r1[lane] = acc1;
      pt[lane * PT + i0] = acc0;
      pt[lane * PT + i0 + 1] = acc1;
    }
    __syncthreads();
    // the trailing lower triangle -= panel panel^T, 4 x 4 tiles
    const int base = b + kCholSub, nt = (NB - base) / 4;
    for (int t = tid; t < nt * nt; t += blockDim.x) {
      const int ti = t / nt, tj = t % nt;
      if (ti < tj) continue;
      const int i0 = base + 4 * ti, c0 = base + 4 * tj;
      double acc[4][4] = {};
#pragma unroll 4
      for (int q = 0; q < kCholSub; ++q) {
        const double2 a01 = *reinterpret_cast<const double2 *>(pt + q * PT + i0);
        const double2 a23 = *reinterpret_cast<const double2 *>(pt + q * PT + i0 + 2);
        const double2 b01 = *reinterpret_cast<const double2 *>(pt + q * PT + c0);
        const double2 b23 = *reinterpret_cast<const double2 *>(pt + q * PT + c0 + 2);
        const double av[4] = {a01.x, a01.y, a23.x, a23.y};
        const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int w = 0; w < 4; ++w) acc[u][w] = fma(av[u], bv[w], acc[u][w]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) s[(i0 + u) * ST + c0 + w] -= acc[u][w];
    }
    __syncthreads();
  }
  // X by block rows: T_ik = sum_{k <= j < i} L_ij X_jk, then X_ik = -X_ii T_ik;
  // each of the 16 warps two rows (warp, warp + 16) of every block, the lanes
  // on columns
  for (int i = 1; i < NB / kCholSub; ++i) {
    const double *l0 = s + (i * kCholSub + warp) * ST;
    const double *l1 = l0 + 16 * ST;
    for (int k = 0; k < i; ++k) {
      double t0 = 0.0, t1 = 0.0;
      const double *xkk = xd + k * kCholSub * XS;
#pragma unroll 8
      for (int q = 0; q < kCholSub; ++q) {
        const double x = xkk[q * XS + lane];
        t0 = fma(l0[k * kCholSub + q], x, t0);
        t1 = fma(l1[k * kCholSub + q], x, t1);
      }
      for (int j = k + 1; j < i; ++j) {
        const double *xc = s + (k * kCholSub + lane) * ST + j * kCholSub;  // X[j*32 + q][k*32 + lane]
#pragma unroll 8
        for (int q = 0; q < kCholSub; ++q) {
          const double x = xc[q];
          t0 = fma(l0[j * kCholSub + q], x, t0);
          t1 = fma(l1[j * kCholSub + q], x, t1);
        }
      }
      tb[(k * kCholSub + warp) * XS + lane] = t0;
      tb[(k * kCholSub + warp + 16) * XS + lane] = t1;
    }
    __syncthreads();
    const double *xii = xd + i * kCholSub * XS;
    for (int k = 0; k < i; ++k) {
      double v0 = 0.0, v1 = 0.0;
#pragma unroll 8
      for (int q = 0; q < kCholSub; ++q) {
        const double tq = tb[(k * kCholSub + q) * XS + lane];
        v0 = fma(xii[warp * XS + q], tq, v0);
        v1 = fma(xii[(warp + 16) * XS + q], tq, v1);
      }
      s[(k * kCholSub + lane) * ST + i * kCholSub + warp] = -v0;
      s[(k * kCholSub + lane) * ST + i * kCholSub + warp + 16] = -v1;
    }
    __syncthreads();
  }
  double *ld = Linv + static_cast<int64_t>(f) * NB * NB;
  for (int i = tid; i < nbj * nbj; i += blockDim.x) {
    const int c = i / nbj, r = i % nbj;
    if (r >= c) a[(j0 + c) * n + j0 + r] = r == c ? diag[c] : s[r * ST + c];
    double x = 0.0;
    if (r == c)
      x = xdiag[c];
    else if (r > c)
      x = (r / kCholSub == c / kCholSub)
              ? xd[(r / kCholSub) * kCholSub * XS + (r % kCholSub) * XS + c % kCholSub]
              : s[c * ST + r];
    ld[c * NB + r] = x;
  }
  if (tid == 0 && bad >= 0 && info[f] == 0) info[f] = static_cast<int>(j0) + bad + 1;
}

// out[r, c] = X[r, p] X[r, c]: the collocation of state p times every
// orbital's, the grid side of the three-index slice B_p = D^T out
__global__ void row_scaled_copy_kernel(const double *__restrict__ X, int64_t M, int64_t n,
                                       int64_t p, double *__restrict__ out) {
  const int64_t total = M * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n;
    out[i] = X[r * n + p] * X[i];
  }
}

// out[p] = sum_P X[P, p] R[P, p] with R in FP32 (a split product's output)
// and X in FP64: the screening contraction's column dots
__global__ void rowdot_f32_kernel(const float *__restrict__ R, int64_t ld_r,
                                  const double *__restrict__ X, int64_t ld_x, int64_t M,
                                  int64_t S, double *out) {
  __shared__ double part[8][33];
  const int64_t p = static_cast<int64_t>(blockIdx.x) * 32 + threadIdx.x;
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 256;
  double s = 0.0;
  if (p < S) {
    const int64_t r1 = min(r0 + 256, M);
    for (int64_t r = r0 + threadIdx.y; r < r1; r += 8)
      s += X[r * ld_x + p] * static_cast<double>(R[r * ld_r + p]);
  }
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && p < S) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x];
    atomicAdd(out + p, t);
  }
}

// out[P, j] = s (C[P, j0 + j] f[j0 + j]) for an nr x nc block of the
// particle-hole columns of C (leading dimension ldc): the explicit response's
// scaled factor, one column chunk at a time
__global__ void cols_scaled_copy_kernel(const double *__restrict__ C, int64_t ldc, int64_t j0,
                                        const double *__restrict__ f, double s, int64_t nr,
                                        int64_t nc, double *__restrict__ out) {
  const int64_t total = nr * nc;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / nc, j = i % nc;
    out[i] = s * (C[r * ldc + j0 + j] * f[j0 + j]);
  }
}

// out[P, q] (+)= factor Y[P, q] v[q] over an nr x nc row-major block
__global__ void col_scale_kernel(const double *__restrict__ Y, const double *__restrict__ v,
                                 int64_t nr, int64_t nc, double factor, double *out,
                                 bool accumulate) {
  const int64_t total = nr * nc;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double x = factor * Y[i] * v[i % nc];
    out[i] = accumulate ? out[i] + x : x;
  }
}

// out[r, c] += a[r * lda + p] b[r, c]: row r scaled by a's column p
__global__ void row_scale_acc_kernel(const double *__restrict__ a, int64_t lda, int64_t p,
                                     const double *__restrict__ b, int64_t nr, int64_t nc,
                                     double *out) {
  const int64_t total = nr * nc;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] += a[(i / nc) * lda + p] * b[i];
}

// out[r * ldo + p] += sum_c G[r, c] X[r, c]: one warp per row
__global__ void row_dot_into_col_kernel(const double *__restrict__ G,
                                        const double *__restrict__ X, int64_t nr, int64_t nc,
                                        double *out, int64_t ldo, int64_t p) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= nr) return;
  double s = 0.0;
  for (int64_t c = lane; c < nc; c += 32) s += G[r * nc + c] * X[r * nc + c];
  for (int d = 16; d; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
  if (lane == 0) out[r * ldo + p] += s;
}

// The batched Cholesky's inverted diagonal blocks of one matrix (block j at
// Linv + j * step_stride, column-major, ld kCholNb) as TF32 pairs in the two
// layouts of the triangular-inverse recursion: rows of L^-1 (r_*) and columns
// of L^-1 as rows (c_*), zeros above the diagonal included, as
// trtri_diag_blocks_kernel writes them. One CTA per block.
__global__ void linv_blocks_to_pairs_kernel(const double *__restrict__ Linv,
                                            int64_t step_stride, int64_t n, float *c_hi,
                                            float *c_lo, float *r_hi, float *r_lo, int64_t ldp) {
  const int64_t off = static_cast<int64_t>(blockIdx.x) * kCholNb;
  const int m = static_cast<int>(min(static_cast<int64_t>(kCholNb), n - off));
  const double *X = Linv + static_cast<int64_t>(blockIdx.x) * step_stride;
  for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
    const int c = idx / m, r = idx % m;
    const double x = X[c * kCholNb + r];
    const float h = to_tf32(static_cast<float>(x));
    const float l = to_tf32(static_cast<float>(x - static_cast<double>(h)));
    r_hi[(off + r) * ldp + off + c] = h;
    r_lo[(off + r) * ldp + off + c] = l;
    c_hi[(off + c) * ldp + off + r] = h;
    c_lo[(off + c) * ldp + off + r] = l;
  }
}

}  // namespace

void launch_chi0_bar_seed(double *a, int64_t n, int nfreq, const double *w, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>(blocks(n * n) / 8 + 1), nfreq);
  count_launch(); chi0_bar_seed_kernel<<<grid, 256, 0, st>>>(a, n, w);
}

void launch_sym_half(const double *in, double *out, int64_t n, cudaStream_t st) {
  count_launch(); sym_half_kernel<<<blocks(n * n), 256, 0, st>>>(in, out, n);
}

void launch_xbar_update(const double *GoX, const double *GvX, const double *X, int64_t M,
                        int64_t n, int64_t nocc, const double *eps, double mu, double tau,
                        double *X_bar, double *eps_bar, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((n + 31) / 32), static_cast<unsigned>((M + 255) / 256));
  count_launch(); xbar_kernel<<<grid, dim3(32, 8), 0, st>>>(GoX, GvX, X, M, n, nocc, eps, mu, tau, X_bar,
                                            eps_bar);
}

void launch_mirror_lower_to_upper(double *a, int64_t n, cudaStream_t st) {
  count_launch(); mirror_kernel<<<blocks(n * n), 256, 0, st>>>(a, n);
}

void launch_lu_logdet(const double *LU, const int *piv, int64_t n, double *logdet, int *sign,
                      cudaStream_t st) {
  count_launch(); lu_logdet_kernel<<<1, 256, 0, st>>>(LU, piv, n, logdet, sign);
}

void launch_diag(double *a, int64_t n, int nmat, double *diag, bool save, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((n + 255) / 256), nmat);
  count_launch(); diag_kernel<<<grid, 256, 0, st>>>(a, n, diag, save);
}

void launch_lower_copy(const double *A, int64_t lda, double *T, int ib, cudaStream_t st) {
  count_launch();
  lower_copy_kernel<<<blocks(static_cast<int64_t>(ib) * ib), 256, 0, st>>>(A, lda, T, ib);
}

void launch_zero_strict_upper_cm(double *a, int64_t n, cudaStream_t st) {
  count_launch();
  zero_strict_upper_cm_kernel<<<blocks(n * n), 256, 0, st>>>(a, n);
}

int launch_trtri_diag_blocks(double *A, int64_t n, int64_t lda, int nb, cudaStream_t st,
                             float *c_hi, float *c_lo, float *r_hi, float *r_lo, int64_t ldp) {
  if (nb < 1 || nb > 128) return MBPT_ERR_SHAPE;  // one thread group of kDiagParts per column
  const size_t smem = sizeof(double) * (static_cast<size_t>(nb) * (nb + 1) + nb);
  // the attribute is per device, so it is set on every call (a host-side write)
  if (cudaFuncSetAttribute(trtri_diag_blocks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return MBPT_ERR_CUDA;
  count_launch();
  trtri_diag_blocks_kernel<<<static_cast<unsigned>((n + nb - 1) / nb), nb * kDiagParts, smem,
                             st>>>(A, n, lda, nb, c_hi, c_lo, r_hi, r_lo, ldp);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

void launch_strided_to_tf32(const double *src, int64_t rows, int64_t k, int64_t rs, int64_t cs,
                            float *hi, float *lo, int64_t rows_p, int64_t k_p, cudaStream_t st) {
  count_launch();
  dim3 grid(static_cast<unsigned>((k_p + 31) / 32), static_cast<unsigned>((rows_p + 31) / 32));
  strided_to_tf32_kernel<<<grid, dim3(32, 8), 0, st>>>(src, rows, k, rs, cs, hi, lo, rows_p,
                                                       k_p);
}

void launch_identity(double *a, int64_t n, cudaStream_t st) {
  count_launch(); identity_kernel<<<blocks(n * n), 256, 0, st>>>(a, n, 0.0, true);
}

void launch_minus_identity(double *a, int64_t n, cudaStream_t st) {
  count_launch(); identity_kernel<<<blocks(n * n), 256, 0, st>>>(a, n, -1.0, false);
}

void launch_sigma_back_gather(const double *X, int64_t M, int64_t n, const int64_t *states,
                              int64_t S, const double *sl, const double *sg, double *Xs,
                              double *Xl, double *Xg, cudaStream_t st) {
  count_launch();
  sigma_back_gather_kernel<<<blocks(M * S), 256, 0, st>>>(X, M, n, states, S, sl, sg, Xs, Xl,
                                                          Xg);
}

void launch_sigma_back_hadamard(double *go, double *gv, double *zt, double *al, double *ag,
                                int64_t total, cudaStream_t st) {
  count_launch();
  sigma_back_hadamard_kernel<<<blocks(total), 256, 0, st>>>(go, gv, zt, al, ag, total);
}

void launch_scatter_cols(const double *T, int64_t M, int64_t S, const int64_t *states,
                         double scale, double *X_bar, int64_t n, cudaStream_t st) {
  count_launch();
  scatter_cols_kernel<<<blocks(M * S), 256, 0, st>>>(T, M, S, states, scale, X_bar, n);
}

void launch_chol_copy_panel(const double *A, int64_t n, int64_t j0, int64_t m, int nbj,
                            int nmat, bool one_minus, double *P, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>(blocks(m * nbj)), nmat);
  count_launch();
  chol_copy_panel_kernel<<<grid, 256, 0, st>>>(A, n, j0, m, nbj, one_minus, P);
}

int launch_chol_diag_block(const double *P, int64_t m, int nbj, double *A, int64_t n,
                           int64_t j0, int nmat, double *Linv, int *info, cudaStream_t st) {
  if (nbj < 1 || nbj > kCholNb) return MBPT_ERR_SHAPE;
  const size_t smem = sizeof(double) * kCholSmemDoubles;
  if (cudaFuncSetAttribute(chol_diag_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return MBPT_ERR_CUDA;
  count_launch();
  chol_diag_block_kernel<<<nmat, 512, smem, st>>>(P, m, nbj, A, n, j0, Linv, info);
  return MBPT_OK;
}

void launch_row_scaled_copy(const double *X, int64_t M, int64_t n, int64_t p, double *out,
                            cudaStream_t st) {
  count_launch();
  row_scaled_copy_kernel<<<blocks(M * n), 256, 0, st>>>(X, M, n, p, out);
}

void launch_rowdot_f32(const float *R, int64_t ld_r, const double *X, int64_t ld_x, int64_t M,
                       int64_t S, double *out, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((S + 31) / 32), static_cast<unsigned>((M + 255) / 256));
  count_launch();
  rowdot_f32_kernel<<<grid, dim3(32, 8), 0, st>>>(R, ld_r, X, ld_x, M, S, out);
}

void launch_cols_scaled_copy(const double *C, int64_t ldc, int64_t j0, const double *f,
                             double s, int64_t nr, int64_t nc, double *out, cudaStream_t st) {
  count_launch();
  cols_scaled_copy_kernel<<<blocks(nr * nc), 256, 0, st>>>(C, ldc, j0, f, s, nr, nc, out);
}

void launch_col_scale(const double *Y, const double *v, int64_t nr, int64_t nc, double factor,
                      double *out, bool accumulate, cudaStream_t st) {
  count_launch();
  col_scale_kernel<<<blocks(nr * nc), 256, 0, st>>>(Y, v, nr, nc, factor, out, accumulate);
}

void launch_row_scale_acc(const double *a, int64_t lda, int64_t p, const double *b, int64_t nr,
                          int64_t nc, double *out, cudaStream_t st) {
  count_launch();
  row_scale_acc_kernel<<<blocks(nr * nc), 256, 0, st>>>(a, lda, p, b, nr, nc, out);
}

void launch_row_dot_into_col(const double *G, const double *X, int64_t nr, int64_t nc,
                             double *out, int64_t ldo, int64_t p, cudaStream_t st) {
  count_launch();
  row_dot_into_col_kernel<<<static_cast<unsigned>((nr + 7) / 8), 256, 0, st>>>(G, X, nr, nc,
                                                                              out, ldo, p);
}

void launch_linv_blocks_to_pairs(const double *Linv, int64_t step_stride, int64_t n,
                                 float *c_hi, float *c_lo, float *r_hi, float *r_lo,
                                 int64_t ldp, cudaStream_t st) {
  count_launch();
  linv_blocks_to_pairs_kernel<<<static_cast<unsigned>((n + kCholNb - 1) / kCholNb), 256, 0,
                                st>>>(Linv, step_stride, n, c_hi, c_lo, r_hi, r_lo, ldp);
}

}  // namespace mbpt
