// Batched Thiele-Pade continuation and quasiparticle root search, one thread
// per state, FP64. Compiled without FMA contraction so that each complex
// operation rounds as the plain expression does.
//
// Per state p (MBPTcode: GW/qp_solve.py:529-558, :575-695):
//   * sample points z = mu +/- i w (occupied states on the negative branch,
//     with Sigma conjugated, qp_solve.py:659, :698-703);
//   * greedy Thiele ordering (analytic_continuation.py:34-61): start at the
//     point nearest the origin, then repeatedly add the point whose next
//     reciprocal-difference coefficient is smallest in magnitude. The
//     candidate's coefficient only needs the new row of the table, computed
//     from the coefficients already chosen;
//   * root of f(w) = w - eps_p - xc_p - Re Sigma(w) (qp_equation.py:1353-1393):
//     150-point scan per window (tiers +-0.5/+-1/+-2 Ha by |eps_p|), slow cells
//     halved up to 6 times, bisection to 1e-8, Z from a central difference
//     (h = 1e-3), the root of largest valid Z; Z > 1/2 ends the search.
//   * optional warm start: safeguarded Newton on the analytic derivative of
//     the continued fraction from a predicted root, accepted only when it
//     converges inside the narrowest window with Z in (1/2, 1]; otherwise
//     the scan above runs as the fallback.
#include <cmath>

#include "common.cuh"

namespace mbpt {
namespace {

constexpr int kMaxPade = 32;
constexpr int kMaxFound = 96;
constexpr int kNOmega = 150;
constexpr double kTol = 1e-8;
constexpr int kMaxBisect = 100;
constexpr double kZStep = 1e-3;
constexpr double kZMin = 0.5;
constexpr double kSecantMin = 0.5;
constexpr int kSplitDepth = 6;
__constant__ double kTierDepth[3] = {0.0, 1.5, 4.0};
__constant__ double kTierHalf[3] = {0.5, 1.0, 2.0};

struct cplx {
  double re, im;
};

__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// Smith's algorithm (Comm. ACM 5, 435 (1962)) for a / b.
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  const double ar = fabs(b.re), ai = fabs(b.im);
  if (ar >= ai) {
    if (ar == 0.0 && ai == 0.0) return {a.re / ar, a.im / ai};
    const double rat = b.im / b.re;
    const double scl = 1.0 / (b.re + b.im * rat);
    return {(a.re + a.im * rat) * scl, (a.im - a.re * rat) * scl};
  }
  const double rat = b.re / b.im;
  const double scl = 1.0 / (b.im + b.re * rat);
  return {(a.re * rat + a.im) * scl, (a.im * rat - a.re) * scl};
}

__device__ __forceinline__ bool cfinite(cplx a) { return isfinite(a.re) && isfinite(a.im); }

struct State {
  cplx z[kMaxPade];  // nodes in greedy order
  cplx a[kMaxPade];  // Thiele coefficients
  int n;
  double eps, xc;
  int evals;
};

// Re of the continued fraction at real w
__device__ double pade_re(const State &s, double w) {
  cplx r = s.a[s.n - 1];
  for (int i = s.n - 2; i >= 0; --i) {
    const cplx d = {w - s.z[i].re, 0.0 - s.z[i].im};
    const cplx t = cmul(d, r);
    r = cdiv(s.a[i], {1.0 + t.re, t.im});
  }
  return r.re;
}

// value and w-derivative of Re of the fraction (forward mode)
__device__ void pade_re_d(const State &s, double w, double &val, double &der) {
  cplx r = s.a[s.n - 1], dr = {0.0, 0.0};
  for (int i = s.n - 2; i >= 0; --i) {
    const cplx d = {w - s.z[i].re, 0.0 - s.z[i].im};
    const cplx t = cmul(d, r);
    const cplx den = {1.0 + t.re, t.im};
    const cplx nr = cdiv(s.a[i], den);
    // d/dw [a / (1 + d r)] = -a (r + d dr) / den^2
    const cplx inner = cmul(d, dr);
    const cplx num = {r.re + inner.re, r.im + inner.im};
    const cplx q = cdiv(cdiv(num, den), den);
    const cplx ndr = cmul({-s.a[i].re, -s.a[i].im}, q);
    r = nr;
    dr = ndr;
  }
  val = r.re;
  der = dr.re;
}

__device__ __forceinline__ double residual(State &s, double w) {
  s.evals++;
  return w - s.eps - s.xc - pade_re(s, w);
}

__device__ double pole_strength(State &s, double w) {
  const double d = (residual(s, w + kZStep) - residual(s, w - kZStep)) / (2.0 * kZStep);
  if (d == 0.0 || !isfinite(d)) return NAN;
  return 1.0 / d;
}

__device__ __forceinline__ bool valid_z(double z, double zmin) {
  return isfinite(z) && zmin < z && z <= 1.0;
}

// bisection of (a, b) as the reference refines a bracket (a = right end)
__device__ double refine(State &s, double a, double b) {
  double fa = residual(s, a);
  for (int it = 0; it < kMaxBisect; ++it) {
    const double c = 0.5 * (a + b);
    const double fc = residual(s, c);
    if (fa * fc <= 0.0) {
      b = c;
    } else {
      a = c;
      fa = fc;
    }
    if (fabs(b - a) <= kTol) break;
  }
  return 0.5 * (a + b);
}

struct Found {
  double w[kMaxFound];
  double z[kMaxFound];
  int n;
  bool overflow;
};

__device__ void solve_bracket(State &s, double l, double r, double fl, double fr, Found &fd) {
  double w;
  if (l == r) {
    w = l;
  } else {
    w = refine(s, r, l);
    const double fw = residual(s, w);
    if (!(fabs(fw) <= fmax(fabs(fl), fabs(fr)))) return;  // a pole, not a root
  }
  if (fd.n >= kMaxFound) {
    fd.overflow = true;
    return;
  }
  fd.w[fd.n] = w;
  fd.z[fd.n] = pole_strength(s, w);
  fd.n++;
}

// brackets of one grid cell, left to right (halving slow cells)
__device__ void cell_brackets(State &s, double l, double r, double fl, double fr, Found &fd) {
  struct Item {
    double l, r, fl, fr;
    int depth;
  };
  Item stack[kSplitDepth + 2];
  int top = 0;
  stack[top++] = {l, r, fl, fr, kSplitDepth};
  while (top > 0) {
    const Item it = stack[--top];
    if (it.fl * it.fr < 0.0) {
      solve_bracket(s, it.l, it.r, it.fl, it.fr, fd);
      continue;
    }
    if (it.depth == 0 || it.fl == 0.0 || it.fr == 0.0 ||
        !(it.fr - it.fl < kSecantMin * (it.r - it.l)))
      continue;
    const double m = 0.5 * (it.l + it.r);
    const double fm = residual(s, m);
    stack[top++] = {m, it.r, fm, it.fr, it.depth - 1};  // right half after the left
    stack[top++] = {it.l, m, it.fl, fm, it.depth - 1};
  }
}

__device__ int select_largest(const Found &fd) {
  int k = -1;
  for (int i = 0; i < fd.n; ++i)
    if (valid_z(fd.z[i], 0.0) && (k < 0 || fd.z[i] > fd.z[k])) k = i;
  return k;
}

// flags: 1 quasiparticle, 2 no root, 4 Z outside (0,1], 8 Pade failed,
//        16 warm start accepted, 32 bracket list overflow
// Thiele coefficients of state i (sample points mu +/- i w, Sigma conjugated
// on the occupied branch) into s.z / s.a, greedily ordered unless greedy is 0;
// false when the greedy ordering finds no finite next coefficient.
__device__ bool build_fit(State &s, const double *sigma, const double *pade_freq, int npade,
                          int i, int64_t p, int64_t nocc, double mu, int greedy) {
  const double sign = p < nocc ? -1.0 : 1.0;
  const bool conj = p < nocc;
  s.n = npade;
  cplx zz[kMaxPade], ff[kMaxPade];
  for (int k = 0; k < npade; ++k) {
    zz[k] = {mu, sign * pade_freq[k]};
    const double re = sigma[2 * (static_cast<int64_t>(i) * npade + k)];
    const double im = sigma[2 * (static_cast<int64_t>(i) * npade + k) + 1];
    ff[k] = {re, conj ? -im : im};
  }
  // ---- Thiele coefficients, greedy order ----
  if (greedy) {
    bool used[kMaxPade];
    int start = 0;
    double best_abs = INFINITY;
    for (int k = 0; k < npade; ++k) {
      used[k] = false;
      const double m = hypot(zz[k].re, zz[k].im);
      if (m < best_abs) {
        best_abs = m;
        start = k;
      }
    }
    used[start] = true;
    s.z[0] = zz[start];
    s.a[0] = ff[start];
    for (int m = 1; m < npade; ++m) {
      int best_j = -1;
      double best = INFINITY;
      cplx best_g = {0.0, 0.0};
      for (int j = 0; j < npade; ++j) {
        if (used[j]) continue;
        cplx g = ff[j];
        for (int q = 1; q <= m; ++q) {
          const cplx dz = {zz[j].re - s.z[q - 1].re, zz[j].im - s.z[q - 1].im};
          const cplx num = {s.a[q - 1].re - g.re, s.a[q - 1].im - g.im};
          g = cdiv(num, cmul(dz, g));
        }
        const double score = hypot(g.re, g.im);
        if (isfinite(score) && score < best) {
          best = score;
          best_j = j;
          best_g = g;
        }
      }
      if (best_j < 0) {
        return false;
      }
      used[best_j] = true;
      s.z[m] = zz[best_j];
      s.a[m] = best_g;
    }
  } else {
    // natural order: the same recursion over the points as given
    for (int m = 0; m < npade; ++m) {
      cplx g = ff[m];
      for (int q = 1; q <= m; ++q) {
        const cplx dz = {zz[m].re - zz[q - 1].re, zz[m].im - zz[q - 1].im};
        const cplx num = {s.a[q - 1].re - g.re, s.a[q - 1].im - g.im};
        g = cdiv(num, cmul(dz, g));
      }
      s.z[m] = zz[m];
      s.a[m] = g;
    }
  }
  return true;
}

__global__ void pade_qp_kernel(const double *sigma, const double *pade_freq, int npade,
                               const double *eps_anchor, const double *xc,
                               const int64_t *states, int nstates, int64_t nocc, double mu,
                               int greedy, const double *warm, double *roots, double *zout,
                               int *flags, int *evals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nstates) return;
  State s;
  const int64_t p = states[i];
  s.eps = eps_anchor[p];
  s.xc = xc ? xc[i] : 0.0;
  s.evals = 0;
  int fl = 0;
  if (!build_fit(s, sigma, pade_freq, npade, i, p, nocc, mu, greedy)) fl |= 8;
  if (fl & 8) {
    roots[i] = NAN;
    zout[i] = NAN;
    flags[i] = fl;
    evals[i] = 0;
    return;
  }
  const double a = s.eps;
  int tier = 0;
  for (int k = 0; k < 3; ++k)
    if (fabs(a) > kTierDepth[k]) tier = k;

  // ---- warm start: safeguarded Newton inside the narrowest window ----
  if (warm) {
    const double lo = a - kTierHalf[tier], hi = a + kTierHalf[tier];
    double w = warm[i];
    bool conv = false;
    if (isfinite(w) && w > lo && w < hi) {
      for (int it = 0; it < 30; ++it) {
        double pv, pd;
        pade_re_d(s, w, pv, pd);
        s.evals++;
        const double f = w - s.eps - s.xc - pv;
        const double fp = 1.0 - pd;
        if (!(fp > 0.0) || !isfinite(f)) break;
        double step = f / fp;
        if (fabs(step) > 0.1) step = copysign(0.1, step);
        w -= step;
        if (!(w > lo && w < hi)) break;
        if (fabs(step) < 1e-12 * fmax(1.0, fabs(w))) {
          conv = true;
          break;
        }
      }
    }
    if (conv) {
      const double z = pole_strength(s, w);
      if (valid_z(z, kZMin)) {
        roots[i] = w;
        zout[i] = z;
        flags[i] = fl | 1 | 16;
        evals[i] = s.evals;
        return;
      }
    }
  }

  // ---- graphical scan ----
  Found fd;
  fd.overflow = false;
  int k = -1;
  double root = NAN, zr = NAN;
  bool done = false;
  for (int t = tier; t < 3 && !done; ++t) {
    const double lo = a - kTierHalf[t], hi = a + kTierHalf[t];
    fd.n = 0;
    const double step = (hi - lo) / (kNOmega - 1);
    double gprev = lo, fprev = residual(s, lo);
    for (int q = 1; q < kNOmega; ++q) {
      const double g = (q == kNOmega - 1) ? hi : static_cast<double>(q) * step + lo;
      const double fg = residual(s, g);
      cell_brackets(s, gprev, g, fprev, fg, fd);
      gprev = g;
      fprev = fg;
    }
    k = select_largest(fd);
    if (k >= 0 && valid_z(fd.z[k], kZMin)) {
      root = fd.w[k];
      zr = fd.z[k];
      fl |= 1;
      done = true;
    }
  }
  if (!done) {
    if (fd.n == 0) {
      fl |= 2;
    } else {
      if (k < 0) {
        k = 0;
        for (int q = 1; q < fd.n; ++q)
          if (fabs(fd.w[q] - a) < fabs(fd.w[k] - a)) k = q;
      }
      root = fd.w[k];
      zr = fd.z[k];
    }
  }
  if (isfinite(root) && !(0.0 < zr && zr <= 1.0)) fl |= 4;
  if (fd.overflow) fl |= 32;
  roots[i] = root;
  zout[i] = zr;
  flags[i] = fl;
  evals[i] = s.evals;
}

// out[i, q] = Re Sigma_c(query[i, q]) of state i's continuation (NaN when its
// Pade construction failed)
__global__ void pade_eval_kernel(const double *sigma, const double *pade_freq, int npade,
                                 const int64_t *states, int nstates, int64_t nocc, double mu,
                                 int greedy, const double *query, int nq, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nstates) return;
  State s;
  s.eps = 0.0;
  s.xc = 0.0;
  s.evals = 0;
  const bool ok = build_fit(s, sigma, pade_freq, npade, i, states[i], nocc, mu, greedy);
  for (int q = 0; q < nq; ++q) {
    const int64_t o = static_cast<int64_t>(i) * nq + q;
    out[o] = ok ? pade_re(s, query[o]) : NAN;
  }
}

}  // namespace

int launch_pade_eval(const double *sigma, const double *pade_freq, int npade,
                     const int64_t *states, int nstates, int64_t nocc, double mu, int greedy,
                     const double *query, int nq, double *out, cudaStream_t st) {
  if (npade < 2 || npade > kMaxPade || nstates < 0 || nq < 1) return MBPT_ERR_SHAPE;
  if (nstates == 0) return MBPT_OK;
  count_launch();
  pade_eval_kernel<<<(nstates + 63) / 64, 64, 0, st>>>(sigma, pade_freq, npade, states,
                                                       nstates, nocc, mu, greedy, query, nq,
                                                       out);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int launch_pade_qp(const double *sigma, const double *pade_freq, int npade,
                   const double *eps_anchor, const double *xc, const int64_t *states,
                   int nstates, int64_t nocc, double mu, int greedy, const double *warm,
                   double *roots, double *z, int *flags, int *evals, cudaStream_t st) {
  if (npade < 2 || npade > kMaxPade || nstates < 0) return MBPT_ERR_SHAPE;
  if (nstates == 0) return MBPT_OK;
  count_launch(); pade_qp_kernel<<<(nstates + 63) / 64, 64, 0, st>>>(sigma, pade_freq, npade, eps_anchor, xc,
                                                     states, nstates, nocc, mu, greedy, warm,
                                                     roots, z, flags, evals);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

}  // namespace mbpt
