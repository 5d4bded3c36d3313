// Kernels of the contour-deformation self-energy evaluated for many
// (state, real frequency) points at once: the imaginary-axis integral term
// with its slope, and the representability test of real frequencies on an
// imaginary-time grid.
#include <cmath>

#include "internal.h"

namespace mbpt {
namespace {

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ void block_sum2(double &a, double &b) {
  __shared__ double sa[32], sb[32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sa[warp] = a;
    sb[warp] = b;
  }
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  a = threadIdx.x < nw ? sa[threadIdx.x] : 0.0;
  b = threadIdx.x < nw ? sb[threadIdx.x] : 0.0;
  if (warp == 0)
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
}

// One block per query j (state slot s_j, real frequency w_j). The integral
// of the Lorentzian kernel g(d, nu) = d / (d^2 + nu^2), d = w - eps_q, against
// wc_s[nu, q] is the Gauss-Legendre sum over the nodes nu_k plus a correction
// for the kernel's singular part: wc(0) (extrapolated linearly in nu^2 from
// the two nodes k1, k2 nearest zero, coefficients e1, e2) times the exact
// integral of g(d, nu) a^2 / (a^2 + nu^2) over nu in [0, inf),
// (pi / 2) sign(d) a / (a + |d|), minus its quadrature. Per q:
//   A_q   = sum_k w_k g_kq wc_kq,      E_q = (pi/2) s_q a/(a+|d|) - sum_k h_k g_kq,
//   A'_q  = sum_k w_k g'_kq wc_kq,     E'_q = -(pi/2) a/(a+|d|)^2 - sum_k h_k g'_kq,
// h_k = w_k a^2 / (a^2 + nu_k^2), g' = dg/dd = (nu^2 - d^2) / (d^2 + nu^2)^2,
// s_q = sign(d) (0 within on_tol of a pole on the contour). The term is
// -(1/pi) sum_q [A_q + E_q (e1 wc_k1q + e2 wc_k2q)] and its slope in w the
// same with the primed parts.
__global__ void cd_integral_kernel(const double *__restrict__ wc, int nfreq, int norb,
                                   const double *__restrict__ eps,
                                   const double *__restrict__ nu,
                                   const double *__restrict__ nu_w, int k1, int k2, double e1,
                                   double e2, double a, double on_tol,
                                   const int *__restrict__ slot,
                                   const double *__restrict__ omega, double *__restrict__ value,
                                   double *__restrict__ slope) {
  const int j = blockIdx.x;
  const double w = omega[j];
  const double *W = wc + static_cast<int64_t>(slot[j]) * nfreq * norb;
  double v = 0.0, dv = 0.0;
  for (int q = threadIdx.x; q < norb; q += blockDim.x) {
    const double d = w - eps[q];
    double A = 0.0, dA = 0.0, H = 0.0, dH = 0.0;
    for (int k = 0; k < nfreq; ++k) {
      const double n2 = nu[k] * nu[k];
      const double den = d * d + n2;
      const double g = d / den;
      const double dg = (n2 - d * d) / (den * den);
      const double x = W[static_cast<int64_t>(k) * norb + q];
      A += nu_w[k] * g * x;
      dA += nu_w[k] * dg * x;
      const double h = nu_w[k] * a * a / (a * a + n2);
      H += h * g;
      dH += h * dg;
    }
    const double ad = a + fabs(d);
    const double side = fabs(d) < on_tol ? 0.0 : (d > 0.0 ? 1.0 : -1.0);
    const double E = 0.5 * kPi * side * a / ad - H;
    const double dE = -0.5 * kPi * a / (ad * ad) - dH;
    const double w0 = e1 * W[static_cast<int64_t>(k1) * norb + q] +
                      e2 * W[static_cast<int64_t>(k2) * norb + q];
    v += A + E * w0;
    dv += dA + dE * w0;
  }
  block_sum2(v, dv);
  if (threadIdx.x == 0) {
    value[j] = -v / kPi;
    slope[j] = -dv / kPi;
  }
}

// One block per real frequency f: max over the pair energies d and both
// signs of y = d -+ f of |y sum_k w_k e^(-y tau_k) - 1|, the error of the
// grid's bare Laplace quadrature of 1/y; infinity where some y <= 0 (f at or
// above the particle-hole gap).
__global__ void laplace_error_kernel(const double *__restrict__ d, int64_t npairs,
                                     const double *__restrict__ tau,
                                     const double *__restrict__ tau_w, int ntau,
                                     const double *__restrict__ freq, double *__restrict__ err) {
  const double f = freq[blockIdx.x];
  double worst = 0.0;
  bool below = false;
  for (int64_t i = threadIdx.x; i < npairs; i += blockDim.x) {
    for (int sgn = 0; sgn < 2; ++sgn) {
      const double y = sgn ? d[i] + f : d[i] - f;
      if (!(y > 0.0)) {
        below = true;
        continue;
      }
      double q = 0.0;
      for (int k = 0; k < ntau; ++k) q += tau_w[k] * exp(-y * tau[k]);
      worst = fmax(worst, fabs(q * y - 1.0));
    }
  }
  __shared__ double sw[32];
  __shared__ int sb[32];
  // every lane takes part in every shuffle (no short-circuit around one)
  for (int o = 16; o > 0; o >>= 1) {
    const double w_other = __shfl_down_sync(0xffffffffu, worst, o);
    const int b_other = __shfl_down_sync(0xffffffffu, below ? 1 : 0, o);
    worst = fmax(worst, w_other);
    below = below || b_other != 0;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sw[warp] = worst;
    sb[warp] = below ? 1 : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double m = 0.0;
    int any = 0;
    for (int i = 0; i < nw; ++i) {
      m = fmax(m, sw[i]);
      any |= sb[i];
    }
    err[blockIdx.x] = any ? INFINITY : m;
  }
}

}  // namespace
}  // namespace mbpt

using namespace mbpt;

extern "C" {

int mbpt_cd_integral_terms(const double *wc, int nslots, int nfreq, int64_t norb,
                           const double *eps, const double *nu, const double *nu_w, int k1,
                           int k2, double e1, double e2, double a, double on_tol,
                           const int *slot, const double *omega, int64_t nq, double *value,
                           double *slope, void *stream) {
  if (nslots < 1 || nfreq < 2 || norb < 1 || nq < 0 || k1 < 0 || k2 < 0 || k1 >= nfreq ||
      k2 >= nfreq || norb > INT32_MAX || nq > INT32_MAX)
    return MBPT_ERR_SHAPE;
  if (nq == 0) return MBPT_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  count_launch();
  cd_integral_kernel<<<static_cast<unsigned>(nq), 256, 0, st>>>(
      wc, nfreq, static_cast<int>(norb), eps, nu, nu_w, k1, k2, e1, e2, a, on_tol, slot, omega,
      value, slope);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int mbpt_laplace_representation_error(const double *d, int64_t npairs, const double *tau,
                                       const double *tau_w, int ntau, const double *freq,
                                       int64_t nf, double *err, void *stream) {
  if (npairs < 1 || ntau < 1 || nf < 0 || nf > INT32_MAX) return MBPT_ERR_SHAPE;
  if (nf == 0) return MBPT_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  count_launch();
  laplace_error_kernel<<<static_cast<unsigned>(nf), 256, 0, st>>>(d, npairs, tau, tau_w, ntau,
                                                                  freq, err);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

}  // extern "C"
