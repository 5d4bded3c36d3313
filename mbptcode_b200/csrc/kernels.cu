// Bandwidth-bound kernels of the route: operand preparation (exponential
// scaling of the collocation branches, BF16 splitting with zero padding),
// the FP64 tau <-> omega transforms, Hadamard products, the Dyson helpers
// around the Cholesky factorisation, and small reductions.
#include <cmath>

#include "internal.h"

namespace mbpt {
namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n, int per = kThreads) {
  int64_t b = (n + per - 1) / per;
  return static_cast<int>(b < 1 ? 1 : (b > (1 << 30) ? (1 << 30) : b));
}

template <typename T>
__device__ __forceinline__ float to_f(T x) { return static_cast<float>(x); }

template <typename T>
__global__ void split_pad_kernel(const T *__restrict__ src, int64_t rows, int64_t cols,
                                 int64_t ld_src, float scale, bf16 *__restrict__ hi,
                                 bf16 *__restrict__ lo, int64_t ld_dst, int64_t rows_p,
                                 int64_t cols_p) {
  const int64_t n = rows_p * cols_p;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / cols_p, c = i % cols_p;
    float x = 0.f;
    if (r < rows && c < cols) x = scale * to_f(src[r * ld_src + c]);
    bf16 h, l;
    split_bf16(x, h, l);
    hi[r * ld_dst + c] = h;
    lo[r * ld_dst + c] = l;
  }
}

// hi/lo[r, c] = the BF16 pair of s (src[r, c] f[c]), zero-padded to rows_p x
// cols_p: the explicit response's particle-hole columns scaled by their
// frequency factor on the way into the split engine
__global__ void split_pad_colscale_kernel(const double *__restrict__ src, int64_t rows,
                                          int64_t cols, int64_t ld_src,
                                          const double *__restrict__ f, double s,
                                          bf16 *__restrict__ hi, bf16 *__restrict__ lo,
                                          int64_t ld_dst, int64_t rows_p, int64_t cols_p) {
  const int64_t n = rows_p * cols_p;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / cols_p, c = i % cols_p;
    float x = 0.f;
    if (r < rows && c < cols) x = static_cast<float>(s * (src[r * ld_src + c] * f[c]));
    bf16 h, l;
    split_bf16(x, h, l);
    hi[r * ld_dst + c] = h;
    lo[r * ld_dst + c] = l;
  }
}

// dst[c][r] = src[r][c] through a 32 x 33 shared tile
template <typename T>
__global__ void split_pad_transpose_kernel(const T *__restrict__ src, int64_t rows,
                                           int64_t cols, int64_t ld_src, float scale,
                                           bf16 *__restrict__ hi, bf16 *__restrict__ lo,
                                           int64_t ld_dst, int64_t rows_p, int64_t cols_p) {
  __shared__ float tile[32][33];
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 32, c0 = static_cast<int64_t>(blockIdx.x) * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t r = r0 + k, c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < rows && c < cols) ? scale * to_f(src[r * ld_src + c]) : 0.f;
  }
  __syncthreads();
  // output row = source column, output column = source row
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t orow = c0 + k, ocol = r0 + threadIdx.x;
    if (orow < cols_p && ocol < rows_p) {
      bf16 h, l;
      split_bf16(tile[threadIdx.x][k], h, l);
      hi[orow * ld_dst + ocol] = h;
      lo[orow * ld_dst + ocol] = l;
    }
  }
}

// Y_o[P,i] = X[P,i] e^{(eps_i - mu) tau / 2},  Y_v[P,a] = X[P,nocc+a] e^{-(eps_a - mu) tau / 2}
// so that G_occ = Y_o Y_o^T and G_virt = Y_v Y_v^T; zero padding to Mp rows
// and to the leading dimensions.
__global__ void prep_branches_kernel(const double *__restrict__ X, int64_t M, int64_t n,
                                     int64_t nocc, const double *__restrict__ eps, double mu,
                                     double tau, bf16 *o_hi, bf16 *o_lo, int64_t ld_o,
                                     bf16 *v_hi, bf16 *v_lo, int64_t ld_v, int64_t Mp) {
  const int64_t width = ld_o + ld_v;
  const int64_t total = Mp * width;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / width, c = i % width;
    float x = 0.f;
    if (c < ld_o) {
      if (r < M && c < nocc) x = static_cast<float>(X[r * n + c] * exp(0.5 * (eps[c] - mu) * tau));
      bf16 h, l;
      split_bf16(x, h, l);
      o_hi[r * ld_o + c] = h;
      o_lo[r * ld_o + c] = l;
    } else {
      const int64_t a = c - ld_o;
      if (r < M && a < n - nocc)
        x = static_cast<float>(X[r * n + nocc + a] * exp(-0.5 * (eps[nocc + a] - mu) * tau));
      bf16 h, l;
      split_bf16(x, h, l);
      v_hi[r * ld_v + a] = h;
      v_lo[r * ld_v + a] = l;
    }
  }
}

// The same Y_o, Y_v as TF32 hi/lo pairs in FP32 words (for the TF32x3 products).
__global__ void prep_branches_tf32_kernel(const double *__restrict__ X, int64_t M, int64_t n,
                                          int64_t nocc, const double *__restrict__ eps,
                                          double mu, double tau, float *o_hi, float *o_lo,
                                          int64_t ld_o, float *v_hi, float *v_lo, int64_t ld_v,
                                          int64_t Mp) {
  const int64_t width = ld_o + ld_v;
  const int64_t total = Mp * width;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / width, c = i % width;
    float x = 0.f, h, l;
    if (c < ld_o) {
      if (r < M && c < nocc) x = static_cast<float>(X[r * n + c] * exp(0.5 * (eps[c] - mu) * tau));
      split_tf32(x, h, l);
      o_hi[r * ld_o + c] = h;
      o_lo[r * ld_o + c] = l;
    } else {
      const int64_t a = c - ld_o;
      if (r < M && a < n - nocc)
        x = static_cast<float>(X[r * n + nocc + a] * exp(-0.5 * (eps[nocc + a] - mu) * tau));
      split_tf32(x, h, l);
      v_hi[r * ld_v + a] = h;
      v_lo[r * ld_v + a] = l;
    }
  }
}

// rows x cols (ld_src) FP64 -> TF32 hi/lo pairs, zero padded to rows_p x cols_p
__global__ void split_pad_tf32_kernel(const double *__restrict__ src, int64_t rows,
                                      int64_t cols, int64_t ld_src, float *hi, float *lo,
                                      int64_t ld_dst, int64_t rows_p, int64_t cols_p) {
  const int64_t n = rows_p * cols_p;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / cols_p, c = i % cols_p;
    const float x = (r < rows && c < cols) ? static_cast<float>(src[r * ld_src + c]) : 0.f;
    float h, l;
    split_tf32(x, h, l);
    hi[r * ld_dst + c] = h;
    lo[r * ld_dst + c] = l;
  }
}

// FP64 reference form: Xo_s[P,i] = X[P,i] e^{power (eps_i-mu) tau},
// Xv_s[P,a] = X[P,nocc+a] e^{-power (eps_a-mu) tau}
__global__ void scaled_branches_kernel(const double *__restrict__ X, int64_t M, int64_t n,
                                       int64_t nocc, const double *__restrict__ eps, double mu,
                                       double tau, double power, double *Xo_s, double *Xv_s) {
  const int64_t total = M * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i % n;
    if (c < nocc)
      Xo_s[r * nocc + c] = X[i] * exp(power * (eps[c] - mu) * tau);
    else
      Xv_s[r * (n - nocc) + (c - nocc)] = X[i] * exp(-power * (eps[c] - mu) * tau);
  }
}

__global__ void hadamard_kernel(double *a, const double *__restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    a[i] *= b[i];
}

__global__ void hadamard3_kernel(double *out, const double *__restrict__ a,
                                 const double *__restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = a[i] * b[i];
}

constexpr int kMaxJ = 34;  // largest tabulated minimax grid

// out[j][r, c] = sum_k w[j,k] in[k][r, c] (ACC: added to out); one element
// per thread, the J output sums in registers, so every input element is read
// once and every output written once.
template <typename Tin, bool ACC = false>
__global__ void __launch_bounds__(256) transform_kernel(
    const Tin *__restrict__ in, int64_t in_slice, int64_t ld_in, int64_t rows, int64_t cols,
    const double *__restrict__ w, int J, int K, double *__restrict__ out, int64_t out_slice,
    int64_t ld_out) {
  __shared__ double ws[kMaxJ * kMaxJ];
  for (int i = threadIdx.x; i < J * K; i += blockDim.x) ws[i] = w[i];
  __syncthreads();
  const int64_t total = rows * cols;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols, c = e % cols;
    double acc[kMaxJ];
#pragma unroll
    for (int j = 0; j < kMaxJ; ++j) acc[j] = 0.0;
    const Tin *src = in + r * ld_in + c;
#pragma unroll 2
    for (int k = 0; k < K; ++k) {
      const double x = static_cast<double>(src[k * in_slice]);
#pragma unroll
      for (int j = 0; j < kMaxJ; ++j)
        if (j < J) acc[j] = fma(ws[j * K + k], x, acc[j]);
    }
    const int64_t o = r * ld_out + c;
#pragma unroll
    for (int j = 0; j < kMaxJ; ++j) {
      if (j < J) {
        if constexpr (ACC) {
          out[j * out_slice + o] += acc[j];
        } else {
          out[j * out_slice + o] = acc[j];
        }
      }
    }
  }
}

// The same transform for J = K = N (every transform of the route: the minimax
// grids pair N tau with N omega points), N a compile-time constant: all N
// inputs of an element are loaded before any arithmetic (N loads in flight
// per element), each thread takes two neighbouring columns so that every
// weight read from shared memory feeds two FMAs, and no loop is predicated.
template <typename Tin, int N>
__global__ void __launch_bounds__(256) transform_n_kernel(
    const Tin *__restrict__ in, int64_t in_slice, int64_t ld_in, int64_t rows, int64_t cols,
    const double *__restrict__ w, double *__restrict__ out, int64_t out_slice, int64_t ld_out) {
  __shared__ double ws[N * N];
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) ws[i] = w[i];
  __syncthreads();
  // one pair of columns per thread and no grid-stride loop, so that nothing
  // invites the compiler to keep the N^2 weights in registers across elements
  const int64_t half = (cols + 1) / 2;
  const int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (e >= rows * half) return;
  const int64_t r = e / half, c = 2 * (e % half);
  const bool two = c + 1 < cols;
  const Tin *src = in + r * ld_in + c;
  double x0[N], x1[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    x0[k] = static_cast<double>(src[k * in_slice]);
    x1[k] = two ? static_cast<double>(src[k * in_slice + 1]) : 0.0;
  }
  double *dst = out + r * ld_out + c;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double a0 = 0.0, a1 = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const double wv = ws[j * N + k];
      a0 = fma(wv, x0[k], a0);
      a1 = fma(wv, x1[k], a1);
    }
    dst[j * out_slice] = a0;
    if (two) dst[j * out_slice + 1] = a1;
  }
}

// a <- I - a for each n x n slice; trace[f] = tr(a) before the update.
__global__ void one_minus_kernel(double *a, int64_t n, double *trace) {
  double *m = a + static_cast<int64_t>(blockIdx.y) * n * n;
  const int64_t total = n * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i % n;
    m[i] = (r == c ? 1.0 : 0.0) - m[i];
  }
  (void)trace;
}

__global__ void trace_kernel(const double *a, int64_t n, double *trace) {
  const double *m = a + static_cast<int64_t>(blockIdx.x) * n * n;
  __shared__ double part[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += m[i * n + i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) trace[blockIdx.x] = part[0];
}

// log det = 2 sum log L_ii of each factor
__global__ void logdet_kernel(const double *L, int64_t n, double *logdet) {
  const double *m = L + static_cast<int64_t>(blockIdx.x) * n * n;
  __shared__ double part[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += log(m[i * n + i]);
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) logdet[blockIdx.x] = 2.0 * part[0];
}

// The inverse lives in one triangle (row-major upper = column-major lower):
// mirror it and subtract the identity, giving W - I.
__global__ void symmetrize_minus_identity_kernel(double *a, int64_t n) {
  double *m = a + static_cast<int64_t>(blockIdx.y) * n * n;
  const int64_t total = n * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i % n;
    if (r > c) m[i] = m[c * n + r];
    if (r == c) m[i] -= 1.0;
  }
}

// out[p] += sign * sum_P Xs[P, p] R[P, p]
__global__ void rowdot_kernel(const double *__restrict__ R, int64_t ld_r,
                              const double *__restrict__ Xs, int64_t ld_x, int64_t M, int64_t S,
                              double sign, double *out) {
  __shared__ double part[8][33];
  const int64_t p = static_cast<int64_t>(blockIdx.x) * 32 + threadIdx.x;
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 256;
  double s = 0.0;
  if (p < S) {
    const int64_t r1 = min(r0 + 256, M);
    for (int64_t r = r0 + threadIdx.y; r < r1; r += 8) s += Xs[r * ld_x + p] * R[r * ld_r + p];
  }
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && p < S) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x];
    atomicAdd(out + p, sign * t);
  }
}

__global__ void gather_cols_f32_kernel(const double *X, int64_t M, int64_t n,
                                       const int64_t *states, int64_t S, float *xs,
                                       int64_t ld_xs, int64_t Mp) {
  const int64_t total = Mp * ld_xs;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / ld_xs, c = i % ld_xs;
    xs[i] = (r < M && c < S) ? static_cast<float>(X[r * n + states[c]]) : 0.f;
  }
}

// hi/lo[s][P] = X[P, states[s]] (transposed, padded to Sp x Mp)
__global__ void gather_cols_split_t_kernel(const double *X, int64_t M, int64_t n,
                                           const int64_t *states, int64_t S, bf16 *hi,
                                           bf16 *lo, int64_t ld, int64_t Sp, int64_t Mp) {
  const int64_t total = Sp * Mp;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t s = i / Mp, r = i % Mp;
    const float x = (s < S && r < M) ? static_cast<float>(X[r * n + states[s]]) : 0.f;
    bf16 h, l;
    split_bf16(x, h, l);
    hi[s * ld + r] = h;
    lo[s * ld + r] = l;
  }
}

__global__ void gather_cols_f64_kernel(const double *X, int64_t M, int64_t n,
                                       const int64_t *states, int64_t S, double *xs) {
  const int64_t total = M * S;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / S, c = i % S;
    xs[i] = X[r * n + states[c]];
  }
}

// sigma[s, w] = -1/2 [sum_k C[w,k] (g + l)[k,s] + i sum_k S[w,k] (g - l)[k,s]],
// branch = (l, g) as (2, ntau, nstates); sigma complex interleaved (nstates, npade)
__global__ void sigma_frequency_kernel(const double *branch, int ntau, int nstates,
                                       const double *C, const double *Sn, int npade,
                                       double *sigma) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nstates * npade) return;
  const int s = idx / npade, w = idx % npade;
  const double *l = branch, *g = branch + static_cast<int64_t>(ntau) * nstates;
  double re = 0.0, im = 0.0;
  for (int k = 0; k < ntau; ++k) {
    const double lk = l[k * nstates + s], gk = g[k * nstates + s];
    re += C[w * ntau + k] * (gk + lk);
    im += Sn[w * ntau + k] * (gk - lk);
  }
  sigma[2 * idx] = -0.5 * re;
  sigma[2 * idx + 1] = -0.5 * im;
}

// E_c = (1/2pi) sum_f w_f (logdet_f + tr_f), summed in frequency order
__global__ void energy_sum_kernel(const double *logdet, const double *trace, const double *w,
                                  int nfreq, double *e_c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double e = 0.0;
  for (int f = 0; f < nfreq; ++f) e += w[f] * (logdet[f] + trace[f]);
  *e_c = e / (2.0 * 3.14159265358979323846);
}

inline int grid_cap(int64_t n) {
  const int b = blocks_for(n);
  return b > 148 * 32 ? 148 * 32 : b;
}

}  // namespace

template <typename T>
void launch_split_pad(const T *src, int64_t rows, int64_t cols, int64_t ld_src, float scale,
                      bf16 *hi, bf16 *lo, int64_t ld_dst, int64_t rows_p, int64_t cols_p,
                      bool transpose, cudaStream_t st) {
  if (!transpose) {
    count_launch(); split_pad_kernel<T><<<grid_cap(rows_p * cols_p), kThreads, 0, st>>>(
        src, rows, cols, ld_src, scale, hi, lo, ld_dst, rows_p, cols_p);
  } else {
    // output is cols_p x rows_p
    dim3 grid(static_cast<unsigned>((cols_p + 31) / 32), static_cast<unsigned>((rows_p + 31) / 32));
    count_launch(); split_pad_transpose_kernel<T><<<grid, dim3(32, 8), 0, st>>>(src, rows, cols, ld_src, scale,
                                                                hi, lo, ld_dst, rows_p, cols_p);
  }
}
template void launch_split_pad<double>(const double *, int64_t, int64_t, int64_t, float, bf16 *,
                                       bf16 *, int64_t, int64_t, int64_t, bool, cudaStream_t);
template void launch_split_pad<float>(const float *, int64_t, int64_t, int64_t, float, bf16 *,
                                      bf16 *, int64_t, int64_t, int64_t, bool, cudaStream_t);

void launch_split_pad_colscale(const double *src, int64_t rows, int64_t cols, int64_t ld_src,
                               const double *f, double s, bf16 *hi, bf16 *lo, int64_t ld_dst,
                               int64_t rows_p, int64_t cols_p, cudaStream_t st) {
  count_launch();
  split_pad_colscale_kernel<<<grid_cap(rows_p * cols_p), kThreads, 0, st>>>(
      src, rows, cols, ld_src, f, s, hi, lo, ld_dst, rows_p, cols_p);
}

void launch_prep_branches(const double *X, int64_t M, int64_t n, int64_t nocc,
                          const double *eps, double mu, double tau, bf16 *o_hi, bf16 *o_lo,
                          int64_t ld_o, bf16 *v_hi, bf16 *v_lo, int64_t ld_v, int64_t Mp,
                          cudaStream_t st) {
  count_launch(); prep_branches_kernel<<<grid_cap(Mp * (ld_o + ld_v)), kThreads, 0, st>>>(
      X, M, n, nocc, eps, mu, tau, o_hi, o_lo, ld_o, v_hi, v_lo, ld_v, Mp);
}

void launch_prep_branches_tf32(const double *X, int64_t M, int64_t n, int64_t nocc,
                               const double *eps, double mu, double tau, float *o_hi,
                               float *o_lo, int64_t ld_o, float *v_hi, float *v_lo,
                               int64_t ld_v, int64_t Mp, cudaStream_t st) {
  count_launch();
  prep_branches_tf32_kernel<<<grid_cap(Mp * (ld_o + ld_v)), kThreads, 0, st>>>(
      X, M, n, nocc, eps, mu, tau, o_hi, o_lo, ld_o, v_hi, v_lo, ld_v, Mp);
}

void launch_split_pad_tf32(const double *src, int64_t rows, int64_t cols, int64_t ld_src,
                           float *hi, float *lo, int64_t ld_dst, int64_t rows_p, int64_t cols_p,
                           cudaStream_t st) {
  count_launch();
  split_pad_tf32_kernel<<<grid_cap(rows_p * cols_p), kThreads, 0, st>>>(
      src, rows, cols, ld_src, hi, lo, ld_dst, rows_p, cols_p);
}

void launch_scaled_branches(const double *X, int64_t M, int64_t n, int64_t nocc,
                            const double *eps, double mu, double tau, double power,
                            double *Xo_s, double *Xv_s, cudaStream_t st) {
  count_launch(); scaled_branches_kernel<<<grid_cap(M * n), kThreads, 0, st>>>(X, M, n, nocc, eps, mu, tau,
                                                               power, Xo_s, Xv_s);
}

void launch_hadamard(double *a, const double *b, int64_t n, cudaStream_t st) {
  count_launch(); hadamard_kernel<<<grid_cap(n), kThreads, 0, st>>>(a, b, n);
}

void launch_hadamard3(double *out, const double *a, const double *b, int64_t n,
                      cudaStream_t st) {
  count_launch(); hadamard3_kernel<<<grid_cap(n), kThreads, 0, st>>>(out, a, b, n);
}

template <typename Tin>
void launch_transform(const Tin *in, int64_t in_slice, int64_t ld_in, int64_t rows,
                      int64_t cols, const double *w_dev, int J, int K, double *out,
                      int64_t out_slice, int64_t ld_out, cudaStream_t st) {
  if (J == K) {
    const int64_t elems = rows * ((cols + 1) / 2);
#define MBPT_TRANSFORM_N(NN)                                                                  \
  case NN:                                                                                    \
    count_launch();                                                                           \
    transform_n_kernel<Tin, NN><<<static_cast<unsigned>((elems + 255) / 256), 256, 0, st>>>( \
        in, in_slice, ld_in, rows, cols, w_dev, out, out_slice, ld_out);                      \
    return;
    switch (J) {
      MBPT_TRANSFORM_N(6) MBPT_TRANSFORM_N(8) MBPT_TRANSFORM_N(10) MBPT_TRANSFORM_N(12)
      MBPT_TRANSFORM_N(14) MBPT_TRANSFORM_N(16) MBPT_TRANSFORM_N(18) MBPT_TRANSFORM_N(20)
      MBPT_TRANSFORM_N(22) MBPT_TRANSFORM_N(24) MBPT_TRANSFORM_N(26) MBPT_TRANSFORM_N(28)
      MBPT_TRANSFORM_N(30) MBPT_TRANSFORM_N(32) MBPT_TRANSFORM_N(34)
      default:
        break;
    }
#undef MBPT_TRANSFORM_N
  }
  count_launch(); transform_kernel<Tin><<<grid_cap(rows * cols), 256, 0, st>>>(
      in, in_slice, ld_in, rows, cols, w_dev, J, K, out, out_slice, ld_out);
}
template void launch_transform<double>(const double *, int64_t, int64_t, int64_t, int64_t,
                                       const double *, int, int, double *, int64_t, int64_t,
                                       cudaStream_t);
template void launch_transform<float>(const float *, int64_t, int64_t, int64_t, int64_t,
                                      const double *, int, int, double *, int64_t, int64_t,
                                      cudaStream_t);

void launch_transform_acc(const double *in, int64_t in_slice, int64_t ld_in, int64_t rows,
                          int64_t cols, const double *w_dev, int J, int K, double *out,
                          int64_t out_slice, int64_t ld_out, cudaStream_t st) {
  count_launch(); transform_kernel<double, true><<<grid_cap(rows * cols), 256, 0, st>>>(
      in, in_slice, ld_in, rows, cols, w_dev, J, K, out, out_slice, ld_out);
}


void launch_trace(const double *a, int64_t n, int nmat, double *trace, cudaStream_t st) {
  count_launch(); trace_kernel<<<nmat, 256, 0, st>>>(a, n, trace);
}

void launch_one_minus(double *a, int64_t n, int nmat, double *trace, cudaStream_t st) {
  if (trace) launch_trace(a, n, nmat, trace, st);
  dim3 grid(static_cast<unsigned>(grid_cap(n * n) / 4 + 1), nmat);
  count_launch(); one_minus_kernel<<<grid, kThreads, 0, st>>>(a, n, trace);
}

void launch_logdet_diag(const double *L, int64_t n, int nmat, double *logdet,
                        cudaStream_t st) {
  count_launch(); logdet_kernel<<<nmat, 256, 0, st>>>(L, n, logdet);
}

void launch_symmetrize_minus_identity(double *a, int64_t n, int nmat, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>(grid_cap(n * n) / 4 + 1), nmat);
  count_launch(); symmetrize_minus_identity_kernel<<<grid, kThreads, 0, st>>>(a, n);
}

void launch_rowdot(const double *R, int64_t ld_r, const double *Xs, int64_t ld_x, int64_t M,
                   int64_t S, double sign, double *out, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((S + 31) / 32), static_cast<unsigned>((M + 255) / 256));
  count_launch(); rowdot_kernel<<<grid, dim3(32, 8), 0, st>>>(R, ld_r, Xs, ld_x, M, S, sign, out);
}

void launch_gather_cols_f32(const double *X, int64_t M, int64_t n, const int64_t *states,
                            int64_t S, float *xs, int64_t ld_xs, int64_t Mp, cudaStream_t st) {
  count_launch(); gather_cols_f32_kernel<<<grid_cap(Mp * ld_xs), kThreads, 0, st>>>(X, M, n, states, S, xs,
                                                                    ld_xs, Mp);
}

void launch_gather_cols_split_t(const double *X, int64_t M, int64_t n, const int64_t *states,
                                int64_t S, bf16 *hi, bf16 *lo, int64_t ld, int64_t Sp,
                                int64_t Mp, cudaStream_t st) {
  count_launch(); gather_cols_split_t_kernel<<<grid_cap(Sp * Mp), kThreads, 0, st>>>(X, M, n, states, S, hi,
                                                                     lo, ld, Sp, Mp);
}

void launch_gather_cols_f64(const double *X, int64_t M, int64_t n, const int64_t *states,
                            int64_t S, double *xs, cudaStream_t st) {
  count_launch(); gather_cols_f64_kernel<<<grid_cap(M * S), kThreads, 0, st>>>(X, M, n, states, S, xs);
}

void launch_sigma_frequency(const double *branch, int ntau, int nstates, const double *C,
                            const double *S, int npade, double *sigma, cudaStream_t st) {
  const int total = nstates * npade;
  count_launch(); sigma_frequency_kernel<<<(total + 127) / 128, 128, 0, st>>>(branch, ntau, nstates, C, S,
                                                              npade, sigma);
}

void launch_energy_sum(const double *logdet, const double *trace, const double *w, int nfreq,
                       double *e_c, cudaStream_t st) {
  count_launch(); energy_sum_kernel<<<1, 32, 0, st>>>(logdet, trace, w, nfreq, e_c);
}

}  // namespace mbpt
