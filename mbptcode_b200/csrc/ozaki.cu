// FP64-accurate trailing updates of the batched Cholesky on the int8 tensor
// cores (tcgen05.mma kind::i8, exact int32 accumulation): the Ozaki scheme.
//
// Digit widths: S = 7 and 8 cut signed 7-bit digits (d_s in [-64, 64], base
// 128, as below); S = 6 cuts signed 8-bit digits of base 254 (x = L_rk / 2^e_r,
// t = 127 x, d_1 = rint(t), then t <- 254 (t - d); d_s in [-127, 127], 47 bits
// in all, against 49 for S = 7), whose levels 2..7 take 21 digit products per
// K step instead of 28. Level l weighs 127^-2 254^-(l-2), exact to one
// rounding in FP64; its int32 sums stay exact for K below 2^31 / (6 127^2).
//
// Each row r of the factor L is scaled by 2^-e_r, with 2^e_r >= sqrt(A_rr)
// (|L_rk| <= sqrt(A_rr) for a positive definite A), and cut into S signed
// digits: x = L_rk 2^-e_r, |x| <= 1, x = sum_s d_s 2^-(7s-1) + O(2^-7S),
// d_s in [-64, 64]. A block column of L is cut once, when it is final, into S
// int8 planes (row r, K = column k contiguous). The update of step j,
// P -= L[j0:, :j0] L[j0:j0+nb, :j0]^T, is then
//   sum over levels l = s + t (2 <= l <= S + 1) of 2^(2 - 7l) sum_(s+t=l) D_s D_t^T,
// each level one int32 TMEM accumulator fed by exact 8-bit products (|sum| <=
// S 64^2 K < 2^31 for K below 65 536), combined in FP64 in the epilogue and
// scaled by 2^(e_r + e_c). The terms dropped (s + t > S + 1) have no sign
// preference off the diagonal; on it (a row against itself) their squares
// are all positive, so each step's diagonal entries are taken from an exact
// FP64 row norm instead, which the slicing of each block column accumulates.
//
// Kernel layout: 128 x 64 output tiles (rows r of the panel, 64 of its
// columns), warp 0 the TMA producer (64-byte swizzled boxes of 64 K), warp 1
// the TMEM owner and MMA issuer (the S(S+1)/2 products of a 32-wide K step
// as one MMA per A plane and group of up to four B planes), warps
// 2-5 the epilogue; two pipeline stages of S A-planes and S B-planes; every
// mbarrier wait bounded, as in the split engine.
#include <algorithm>

#include "internal.h"

namespace mbpt {
namespace ozaki {

using umma::mbar_expect_tx;
using umma::mbar_init;
using umma::mbar_wait;
using umma::mma_commit;
using umma::smem_u32;
using umma::tc_fence_after;
using umma::tc_fence_before;

constexpr int BM = 128;   // panel rows per tile
constexpr int BN = 64;    // panel columns per tile
constexpr int BKB = 64;   // K bytes (int8 elements) per stage: two MMA K steps
// (32-byte steps with four stages in the same shared memory measured slower:
// 64.9 against 70.1 TFLOP/s FP64-equivalent at 4096^3)
// the K-major operand layout of a stage's rows: BKB-byte rows swizzled by
// BKB bytes, in 8-row groups of 8 * BKB bytes
constexpr int kSwizzleBytes = BKB;
constexpr CUtensorMapSwizzle kTmaSwizzle =
    kSwizzleBytes == 32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B;
constexpr int kStackPlanes = 4;  // B planes per MMA: N = 4 x 64 = 256, the largest

template <int S>
struct Layout {
  static constexpr int kAPlane = BM * BKB;   // 8 KB
  static constexpr int kBPlane = BN * BKB;   // 4 KB
  static constexpr int kStageBytes = S * (kAPlane + kBPlane);
  // as many stages as 196 KB hold: 2 for S = 7 and 8 (84 and 96 KB each)
  static constexpr int kStages = (196 * 1024) / kStageBytes < 8 ? (196 * 1024) / kStageBytes : 8;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 256;
  static constexpr int kLevels = S;
  static constexpr int kTmemCols = 512;
  static_assert(kLevels * BN <= 512, "levels exceed TMEM");
};

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *tm, int x, int y,
                                            int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// K-major operand with kSwizzleBytes-byte rows and swizzle: 8-row groups
// 8 * kSwizzleBytes bytes apart (layout type 6 = 32-byte swizzle, 4 = 64-byte).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
  static_assert(kSwizzleBytes == 32 || kSwizzleBytes == 64, "32- or 64-byte swizzle");
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>(1) << 16;
  d |= static_cast<uint64_t>((8 * kSwizzleBytes) >> 4) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(kSwizzleBytes == 32 ? 6 : 4) << 61;
  return d;
}

// Instruction descriptor: s8 x s8 -> s32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_s8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_s8(uint32_t tmem_d, uint64_t da, uint64_t db,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tmem_ld32_s32(uint32_t addr, int (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
        "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
        "=r"(v[31])
      : "r"(addr)
      : "memory");
}

enum Epi : int {
  EPI_CHOL = 0,  // the Cholesky panel: P -= product, column-major, exact diagonal
  EPI_GEMM = 1,  // C = alpha product + beta C, row-major
};

struct UpdateArgs {
  CUtensorMap tm_a;    // A digit planes (K, rows, planes), box 64 x 128
  CUtensorMap tm_b;    // B digit planes, box 64 x 64 (the Cholesky: the same array)
  int64_t n;           // matrix size (Cholesky)
  int j0, nb;          // the step's first column and width (<= 128) (Cholesky)
  int k_tiles;         // K / BKB
  int nmat;            // planes per digit level (matrices of a batch)
  int a_row0, b_row0;  // first plane rows of the A and B operands
  int tiles_n;         // 64-column tiles per row of tiles
  double *P;           // nmat panels, column-major m x nb (ld m), m = n - j0
  int64_t p_stride;    // elements between panels
  const double *scale; // Cholesky: nmat x n, 2^e_r; GEMM: the rows of A
  const double *scale_b;  // GEMM: the rows of B
  const double *rowsq; // nmat x n: sum_(k < j0) L_(r, k)^2 of each row, exact
  double *C;           // GEMM output, row-major m_rows x n_cols, ld ldc
  int64_t ldc;
  double alpha, beta;
  int m_rows, n_cols;
  int tiles_m;
  int sym;             // GEMM: symmetric product, upper tiles formed and mirrored
  const double *H1, *H2;  // GEMM: element-wise factors of C and C2 (null: none)
  double *C2;
  int *err;
};

template <int S, int EPI>
__global__ void __launch_bounds__(192, 1) chol_update_kernel(const __grid_constant__ UpdateArgs p) {
  static_assert(S != 6 || EPI == EPI_CHOL, "8-bit digits: the Cholesky's planes only");
  using L = Layout<S>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L::kStages * L::kStageBytes);
  uint64_t *empty = full + L::kStages;
  uint64_t *accum = empty + L::kStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(accum + 1);
  int *fail = reinterpret_cast<int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int f = blockIdx.y;
  const int tm = blockIdx.x / p.tiles_n, tn = blockIdx.x % p.tiles_n;
  const int r0 = tm * BM;       // tile row (Cholesky: matrix row j0 + r0)
  const int c0 = tn * BN;       // tile column
  // uniform: the second half of a narrow last panel, a tile below the
  // diagonal of a symmetric product
  if (EPI == EPI_CHOL && c0 >= p.nb) return;
  if (EPI == EPI_GEMM && p.sym && c0 + BN <= r0) return;
  const int m = static_cast<int>(p.n - p.j0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < L::kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    *fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(L::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      bool ok = true;
      int it = 0;
      for (int kt = 0; kt < p.k_tiles; ++kt, ++it) {
        const int s = it % L::kStages;
        const uint32_t ph = (it / L::kStages) & 1;
        if (!mbar_wait(&empty[s], ph ^ 1)) { ok = false; break; }
        mbar_expect_tx(&full[s], L::kStageBytes);
        uint8_t *st = smem + s * L::kStageBytes;
        const int kx = kt * BKB;
#pragma unroll
        for (int q = 0; q < S; ++q) {
          const int plane = q * p.nmat + f;
          tma_load_3d(st + q * L::kAPlane, &p.tm_a, kx, p.a_row0 + r0, plane, &full[s]);
          tma_load_3d(st + S * L::kAPlane + q * L::kBPlane, &p.tm_b, kx, p.b_row0 + c0, plane,
                      &full[s]);
        }
      }
      if (!ok) {
        atomicExch(fail, 1);
        DevErr{p.err}.set(MBPT_ERR_TIMEOUT);
      }
      for (int q = max(0, it - L::kStages); q < it; ++q)
        mbar_wait(&full[q % L::kStages], (q / L::kStages) & 1);
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      bool ok = true;
      for (int kt = 0; kt < p.k_tiles; ++kt) {
        const int s = kt % L::kStages;
        const uint32_t ph = (kt / L::kStages) & 1;
        if (!mbar_wait(&full[s], ph) || *reinterpret_cast<volatile int *>(fail)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t st = smem_u32(smem + s * L::kStageBytes);
#pragma unroll
        for (int kk = 0; kk < BKB / 32; ++kk) {
          const uint64_t adv = static_cast<uint64_t>(kk * 2);  // 32 bytes >> 4
          const bool first = kt == 0 && kk == 0;
          // A plane sa against the B planes 1 .. S + 1 - sa stacked as one
          // operand (they lie back to back, 64 rows each): product (sa, t)
          // lands in column block sa + t - 2, its level's accumulator, so one
          // MMA of up to 256 columns serves four levels and A is read from
          // shared memory once per four products. Plane 1 covers every
          // level, so its MMAs open the accumulators.
#pragma unroll
          for (int sa = 1; sa <= S; ++sa) {
            const uint64_t da = kmajor_desc(st + (sa - 1) * L::kAPlane) + adv;
#pragma unroll
            for (int t0 = 1; t0 <= S + 1 - sa; t0 += kStackPlanes) {
              const int cnt = S + 1 - sa - t0 + 1 < kStackPlanes ? S + 1 - sa - t0 + 1
                                                                  : kStackPlanes;
              const uint32_t d = tmem + static_cast<uint32_t>((sa - 1 + t0 - 1) * BN);
              const uint64_t db =
                  kmajor_desc(st + S * L::kAPlane + (t0 - 1) * L::kBPlane) + adv;
              mma_s8(d, da, db, idesc_s8(cnt * BN), (first && sa == 1) ? 0u : 1u);
            }
          }
        }
        mma_commit(&empty[s]);
      }
      if (!ok) {
        atomicExch(fail, 1);
        DevErr{p.err}.set(MBPT_ERR_TIMEOUT);
      }
      mma_commit(accum);
      mbar_wait(accum, 0);  // no MMA may still write TMEM when it is freed
    }
    __syncwarp();
  } else {
    const int sp = warp & 3;
    const uint32_t taddr = tmem + (static_cast<uint32_t>(sp * 32) << 16);
    const bool ok = mbar_wait(accum, 0) && !*reinterpret_cast<volatile int *>(fail);
    __syncwarp();
    if (!ok) {
      if (lane == 0) DevErr{p.err}.set(MBPT_ERR_TIMEOUT);
    } else {
      tc_fence_after();
      const int pr = r0 + sp * 32 + lane;             // tile row of this thread
      const bool live = EPI == EPI_CHOL ? pr < m : pr < p.m_rows;
      const int64_t row = EPI == EPI_CHOL ? p.j0 + pr : pr;
      const double *sc = p.scale + (EPI == EPI_CHOL ? static_cast<int64_t>(f) * p.n : 0);
      const double srow = live ? sc[row] : 0.0;
      double *P = EPI == EPI_CHOL ? p.P + static_cast<int64_t>(f) * p.p_stride : nullptr;
#pragma unroll 1
      for (int ch = 0; ch < BN / 32; ++ch) {
        double acc[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[i] = 0.0;
        // smallest levels first
#pragma unroll 1
        for (int lev = S + 1; lev >= 2; --lev) {
          int v[32];
          tmem_ld32_s32(taddr + static_cast<uint32_t>((lev - 2) * BN + ch * 32), v);
          double w;
          if constexpr (S == 6) {
            // 1 / (127^2 254^(lev - 2)): the power is an exact integer below 2^53
            double pw = 16129.0;
            for (int q = 2; q < lev; ++q) pw *= 254.0;
            w = 1.0 / pw;
          } else {
            w = ldexp(1.0, 2 - 7 * lev);
          }
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[i] += static_cast<double>(v[i]) * w;
        }
        if (EPI == EPI_CHOL && live) {
          // all 32 loads first (P's column entries and the columns' scales),
          // then the stores: one memory round trip per chunk instead of one
          // per column, which the compiler cannot reorder across the stores
          // (two halves of 16 columns: the registers hold acc and one half)
          double *Prow = P + pr;   // column pc of the panel at Prow + pc m
          // the diagonal entry from the exact running row norm
          const int pd = pr - c0 - ch * 32;
          const double diag = (pd >= 0 && pd < 32 && pr < p.nb)
                                  ? p.rowsq[static_cast<int64_t>(f) * p.n + p.j0 + pr] : 0.0;
#pragma unroll
          for (int h = 0; h < 32; h += 16) {
            double old[16], scol[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int pc = c0 + ch * 32 + h + i;  // panel column
              old[i] = pc < p.nb ? Prow[static_cast<int64_t>(pc) * m] : 0.0;
              scol[i] = pc < p.nb ? sc[p.j0 + pc] : 0.0;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int pc = c0 + ch * 32 + h + i;
              if (pc < p.nb)
                Prow[static_cast<int64_t>(pc) * m] =
                    pr == pc ? old[i] - diag : old[i] - acc[h + i] * srow * scol[i];
            }
          }
        } else if (EPI == EPI_GEMM && live) {
          const int64_t ro = static_cast<int64_t>(pr) * p.ldc;
          const double a = p.alpha * srow;
          // eight columns at a time: their loads (column scales, factors, the
          // old C) ahead of their stores, one memory round trip per eight
#pragma unroll
          for (int h = 0; h < 32; h += 8) {
            double sb[8], f1[8], f2[8], cold[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const int col = c0 + ch * 32 + h + i;
              const bool in = col < p.n_cols && (!p.sym || col >= pr);
              sb[i] = in ? p.scale_b[col] : 0.0;
              f1[i] = in && p.H1 ? p.H1[ro + col] : 0.0;
              f2[i] = in && p.H1 && p.H2 ? p.H2[ro + col] : 0.0;
              cold[i] = in && !p.H1 && p.beta != 0.0 ? p.C[ro + col] : 0.0;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const int col = c0 + ch * 32 + h + i;
              // symmetric: the upper triangle, each entry also at its mirror
              // (the lanes' rows are consecutive, so the mirrored stores of
              // one column coalesce)
              if (col < p.n_cols && (!p.sym || col >= pr)) {
                const double v = a * acc[h + i] * sb[i];
                const int64_t mo = static_cast<int64_t>(col) * p.ldc + pr;
                const bool mirror = p.sym && col > pr;
                if (p.H1) {
                  const double o1 = v * f1[i];
                  p.C[ro + col] = o1;
                  if (mirror) p.C[mo] = o1;
                  if (p.H2) {
                    const double o2 = v * f2[i];
                    p.C2[ro + col] = o2;
                    if (mirror) p.C2[mo] = o2;
                  }
                } else {
                  const double o = p.beta == 0.0 ? v : v + p.beta * cold[i];
                  p.C[ro + col] = o;
                  if (mirror) p.C[mo] = o;
                }
              }
            }
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(L::kTmemCols)
                 : "memory");
  }
}

// scale[f][r] = 2^e_r with e_r = ceil(log2(sqrt(A_rr))) (A column-major, ld n);
// 1 for a diagonal that is not positive and finite (that matrix fails its
// factorisation and is redone by LU; its digits only need to stay in range).
__global__ void chol_scale_kernel(const double *A, int64_t n, int64_t mat_stride, int nmat,
                                  bool one_minus, double *scale) {
  const int64_t total = n * nmat;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t f = i / n, r = i % n;
    const double d = A[f * mat_stride + r * n + r];
    const double a = one_minus ? 1.0 - d : d;  // the diagonal of I - A_f
    double s = 1.0;
    if (a > 0.0 && a < 1e300) {
      int e;
      frexp(sqrt(a), &e);          // sqrt(a) = m 2^e, m in [0.5, 1): 2^e >= sqrt(a)
      s = ldexp(1.0, e);
    }
    scale[i] = s;
  }
}

// Digits of block column [j0, j0 + nb) of L (column-major in A, ld n, rows
// j0..n-1): plane q of matrix f, row r, K = column c, at
// D[((q * nmat + f) * npad + r) * npad + c]. Rows are read contiguously through
// shared memory and written 16 columns per thread.
template <int S>
__global__ void chol_slice_kernel(const double *A, int64_t n, int64_t mat_stride, int nmat,
                                  int j0, int nb, const double *scale, int8_t *D,
                                  int64_t npad, double *rownorm) {
  __shared__ double tile[32][129];
  const int f = blockIdx.y;
  const int64_t rbase = j0 + static_cast<int64_t>(blockIdx.x) * 32;
  const double *Af = A + f * mat_stride;
  // load 32 rows x nb columns: threads walk rows fastest (column-major source)
  for (int t = threadIdx.x; t < 32 * 128; t += blockDim.x) {
    const int rr = t & 31, cc = t >> 5;
    const int64_t r = rbase + rr;
    // the factor is lower triangular: above the block's diagonal A still holds
    // 1 - chi0, which is not part of L
    tile[rr][cc] = (r < n && cc < nb && r >= j0 + cc)
                       ? Af[static_cast<int64_t>(j0 + cc) * n + r] : 0.0;
  }
  __syncthreads();
  // each thread: one row, 16 consecutive columns, all S planes
  const int rr = threadIdx.x >> 3, cg = (threadIdx.x & 7) * 16;
  const int64_t r = rbase + rr;
  // the rows' running FP64 norms over the columns cut so far (the exact
  // diagonal of the later updates), summed over the 8 threads of a row in a
  // fixed order
  double sq = 0.0;
#pragma unroll
  for (int i = 0; i < 16; ++i) sq = fma(tile[rr][cg + i], tile[rr][cg + i], sq);
  sq += __shfl_xor_sync(0xffffffffu, sq, 1);
  sq += __shfl_xor_sync(0xffffffffu, sq, 2);
  sq += __shfl_xor_sync(0xffffffffu, sq, 4);
  if (r >= n) return;
  if (cg == 0) rownorm[static_cast<int64_t>(f) * n + r] += sq;
  // 7-bit digits: |t| <= 64, base 128; 8-bit (S = 6): |t| <= 127, base 254
  constexpr double kTop = S == 6 ? 127.0 : 64.0, kBase = S == 6 ? 254.0 : 128.0;
  const double inv = kTop / scale[static_cast<int64_t>(f) * n + r];
  __align__(16) int8_t out[S][16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    double t = tile[rr][cg + i] * inv;   // |t| <= kTop
#pragma unroll
    for (int q = 0; q < S; ++q) {
      double d = rint(t);
      d = fmin(fmax(d, -127.0), 127.0);  // non-finite input stays in range
      out[q][i] = static_cast<int8_t>(static_cast<int>(d));
      t = (t - d) * kBase;
    }
  }
  if (cg >= nb) return;
#pragma unroll
  for (int q = 0; q < S; ++q) {
    int8_t *dst = D + ((static_cast<int64_t>(q) * nmat + f) * npad + r) * npad + j0 + cg;
    *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(out[q]);
  }
}


// scale[i] = 2^e >= max_k |x(i, k)| of each row of an operand (1 for a row
// of zeros or with a non-finite entry); x(i, k) = src[i ld + k], or
// src[k ld + i] with trans.
__global__ void row_scale_kernel(const double *src, int64_t rows, int64_t kdim, int64_t ld,
                                 int trans, double *scale) {
  const int lane = threadIdx.x & 31;
  if (trans) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < rows;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      double mx = 0.0;
      for (int64_t k = 0; k < kdim; ++k) mx = fmax(mx, fabs(src[k * ld + i]));
      int e = 0;
      frexp(mx, &e);
      scale[i] = (mx > 0.0 && mx < 1e300) ? ldexp(1.0, e) : 1.0;
    }
    return;
  }
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x >> 5) + (threadIdx.x >> 5);
       i < rows; i += warps) {
    double mx = 0.0;
    for (int64_t k = lane; k < kdim; k += 32) mx = fmax(mx, fabs(src[i * ld + k]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      int e = 0;
      frexp(mx, &e);
      scale[i] = (mx > 0.0 && mx < 1e300) ? ldexp(1.0, e) : 1.0;
    }
  }
}

// Digit planes of an operand (rows x kdim, row scales `scale`): plane q, row
// i, column k at planes[(q rows_pad + i) k_pad + k], zeros beyond rows and
// kdim up to rows_pad and k_pad. One block per 32 rows x 128 columns,
// through shared memory so that both layouts of the source are read along
// their contiguous index.
template <int S>
__global__ void operand_slice_kernel(const double *src, int64_t rows, int64_t kdim, int64_t ld,
                                     int trans, const double *scale, int8_t *planes,
                                     int64_t rows_pad, int64_t k_pad) {
  __shared__ double tile[32][129];
  const int64_t i0 = static_cast<int64_t>(blockIdx.y) * 32;
  const int64_t k0 = static_cast<int64_t>(blockIdx.x) * 128;
  for (int t = threadIdx.x; t < 32 * 128; t += blockDim.x) {
    int rr, kk;
    if (trans) {
      rr = t & 31;
      kk = t >> 5;
    } else {
      rr = t >> 7;
      kk = t & 127;
    }
    const int64_t i = i0 + rr, k = k0 + kk;
    double v = 0.0;
    if (i < rows && k < kdim) v = trans ? src[k * ld + i] : src[i * ld + k];
    tile[rr][kk] = v;
  }
  __syncthreads();
  const int rr = threadIdx.x >> 3, cg = (threadIdx.x & 7) * 16;
  const int64_t i = i0 + rr;
  if (i >= rows_pad) return;
  const double inv = i < rows ? 64.0 / scale[i] : 0.0;
  __align__(16) int8_t out[S][16];
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    double t = tile[rr][cg + c] * inv;     // |t| <= 64
#pragma unroll
    for (int q = 0; q < S; ++q) {
      double d = rint(t);
      d = fmin(fmax(d, -127.0), 127.0);
      out[q][c] = static_cast<int8_t>(static_cast<int>(d));
      t = (t - d) * 128.0;
    }
  }
#pragma unroll
  for (int q = 0; q < S; ++q) {
    int8_t *dst = planes + (static_cast<int64_t>(q) * rows_pad + i) * k_pad + k0 + cg;
    *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(out[q]);
  }
}

bool make_operand_map(CUtensorMap *m, const int8_t *planes, int64_t k_pad, int64_t rows_pad,
                      int64_t nplanes, int box_rows) {
  auto fn = encode_fn();
  if (!fn || (reinterpret_cast<uintptr_t>(planes) & 15) || k_pad % 128) return false;
  cuuint64_t dims[3] = {static_cast<cuuint64_t>(k_pad), static_cast<cuuint64_t>(rows_pad),
                        static_cast<cuuint64_t>(nplanes)};
  cuuint64_t strides[2] = {static_cast<cuuint64_t>(k_pad),
                           static_cast<cuuint64_t>(k_pad * rows_pad)};
  cuuint32_t box[3] = {static_cast<cuuint32_t>(BKB), static_cast<cuuint32_t>(box_rows), 1};
  cuuint32_t es[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t *>(planes), dims, strides,
            box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, kTmaSwizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool make_plane_map(CUtensorMap *m, const int8_t *D, int64_t npad, int64_t planes,
                    int box_rows) {
  auto fn = encode_fn();
  if (!fn || (reinterpret_cast<uintptr_t>(D) & 15) || npad % 128) return false;
  cuuint64_t dims[3] = {static_cast<cuuint64_t>(npad), static_cast<cuuint64_t>(npad),
                        static_cast<cuuint64_t>(planes)};
  cuuint64_t strides[2] = {static_cast<cuuint64_t>(npad),
                           static_cast<cuuint64_t>(npad * npad)};
  cuuint32_t box[3] = {static_cast<cuuint32_t>(BKB), static_cast<cuuint32_t>(box_rows), 1};
  cuuint32_t es[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t *>(D), dims, strides, box,
            es, CU_TENSOR_MAP_INTERLEAVE_NONE, kTmaSwizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline int grid_blocks(int64_t n) {
  int64_t b = (n + 255) / 256;
  return static_cast<int>(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

}  // namespace ozaki

size_t ozaki_planes_bytes(int64_t n, int nmat, int slices) {
  const int64_t npad = round_up(n, 128);
  return static_cast<size_t>(slices) * nmat * npad * npad;
}

int ozaki_chol_scales(const double *A, int64_t n, int nmat, double *scale, double *rownorm,
                      bool one_minus, cudaStream_t st) {
  if (cudaMemsetAsync(rownorm, 0, sizeof(double) * n * nmat, st) != cudaSuccess)
    return MBPT_ERR_CUDA;
  count_launch();
  ozaki::chol_scale_kernel<<<ozaki::grid_blocks(n * nmat), 256, 0, st>>>(A, n, n * n, nmat,
                                                                         one_minus, scale);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int ozaki_chol_slice(const double *A, int64_t n, int nmat, int64_t j0, int nb,
                     const double *scale, int8_t *planes, int slices, double *rownorm,
                     cudaStream_t st) {
  const int64_t npad = round_up(n, 128);
  dim3 grid(static_cast<unsigned>((n - j0 + 31) / 32), nmat);
  count_launch();
  if (slices == 8)
    ozaki::chol_slice_kernel<8><<<grid, 256, 0, st>>>(A, n, n * n, nmat, static_cast<int>(j0),
                                                      nb, scale, planes, npad, rownorm);
  else if (slices == 6)
    ozaki::chol_slice_kernel<6><<<grid, 256, 0, st>>>(A, n, n * n, nmat, static_cast<int>(j0),
                                                      nb, scale, planes, npad, rownorm);
  else if (slices == 7)
    ozaki::chol_slice_kernel<7><<<grid, 256, 0, st>>>(A, n, n * n, nmat, static_cast<int>(j0),
                                                      nb, scale, planes, npad, rownorm);
  else
    return MBPT_ERR_SHAPE;
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int ozaki_chol_update(double *A, int64_t n, int nmat, int64_t j0, int nb, double *P,
                      const double *scale, const int8_t *planes, int slices, double *rowsq,
                      int *err, cudaStream_t st) {
  if (j0 <= 0) return MBPT_OK;
  if (j0 % ozaki::BKB || nb < 1 || nb > 128 || j0 >= 65536 ||
      (slices == 6 && j0 > kOzakiEightBitMaxK))
    return MBPT_ERR_SHAPE;
  const int64_t npad = round_up(n, 128);
  ozaki::UpdateArgs p{};
  if (!ozaki::make_plane_map(&p.tm_a, planes, npad, static_cast<int64_t>(slices) * nmat,
                             ozaki::BM) ||
      !ozaki::make_plane_map(&p.tm_b, planes, npad, static_cast<int64_t>(slices) * nmat,
                             ozaki::BN))
    return MBPT_ERR_SHAPE;
  const int64_t m = n - j0;
  p.n = n;
  p.j0 = static_cast<int>(j0);
  p.nb = nb;
  p.k_tiles = static_cast<int>(j0 / ozaki::BKB);
  p.nmat = nmat;
  p.P = P;
  p.p_stride = m * nb;
  p.scale = scale;
  p.rowsq = rowsq;
  p.tiles_m = static_cast<int>((m + ozaki::BM - 1) / ozaki::BM);
  p.a_row0 = p.b_row0 = static_cast<int>(j0);
  p.tiles_n = 2;
  p.scale_b = nullptr;
  p.C = nullptr;
  p.ldc = 0;
  p.alpha = p.beta = 0.0;
  p.m_rows = p.n_cols = 0;
  p.err = err;
  const dim3 grid(static_cast<unsigned>(p.tiles_m * 2), nmat);
  static std::atomic<uint64_t> attr8{0}, attr7{0}, attr6{0};
  if (slices == 6) {
    auto kern = ozaki::chol_update_kernel<6, ozaki::EPI_CHOL>;
    const int smem = ozaki::Layout<6>::kSmemBytes;
    if (!allow_smem(reinterpret_cast<const void *>(kern), smem, attr6)) return MBPT_ERR_CUDA;
    count_launch();
    kern<<<grid, 192, smem, st>>>(p);
  } else if (slices == 8) {
    auto kern = ozaki::chol_update_kernel<8, ozaki::EPI_CHOL>;
    const int smem = ozaki::Layout<8>::kSmemBytes;
    if (!allow_smem(reinterpret_cast<const void *>(kern), smem, attr8)) return MBPT_ERR_CUDA;
    count_launch();
    kern<<<grid, 192, smem, st>>>(p);
  } else if (slices == 7) {
    auto kern = ozaki::chol_update_kernel<7, ozaki::EPI_CHOL>;
    const int smem = ozaki::Layout<7>::kSmemBytes;
    if (!allow_smem(reinterpret_cast<const void *>(kern), smem, attr7)) return MBPT_ERR_CUDA;
    count_launch();
    kern<<<grid, 192, smem, st>>>(p);
  } else {
    return MBPT_ERR_SHAPE;
  }
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// ---- the general FP64-accurate GEMM ------------------------------------------
// Largest K of one product pass: S 64^2 K must stay below 2^31 (S <= 8).

size_t ozaki_gemm_scratch_bytes(int64_t m, int64_t n, int64_t k, int slices) {
  const int64_t kc = std::min<int64_t>(round_up(k, 128), kOzakiKChunk);
  const int64_t mp = round_up(m, 128), np = round_up(n, 128);
  return static_cast<size_t>(slices) * (mp + np) * kc + 8 * (mp + np) + 4096;
}

int ozaki_dgemm(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha,
                const double *A, int64_t lda, const double *B, int64_t ldb, double beta,
                double *C, int64_t ldc, int slices, void *scratch, size_t scratch_bytes,
                int *err, cudaStream_t st, const OzakiEpi *epi) {
  if (m < 1 || n < 1 || k < 1) return MBPT_ERR_SHAPE;
  if (slices != 7 && slices != 8) return MBPT_ERR_SHAPE;
  const OzakiEpi none;
  const OzakiEpi &x = epi ? *epi : none;
  if (x.sym && m != n) return MBPT_ERR_SHAPE;
  if (x.h1 && (beta != 0.0 || k > kOzakiKChunk || (x.h2 && !x.c2))) return MBPT_ERR_SHAPE;
  if (scratch_bytes < ozaki_gemm_scratch_bytes(m, n, k, slices)) return MBPT_ERR_WORKSPACE;
  const int64_t mp = round_up(m, 128), np = round_up(n, 128);
  static std::atomic<uint64_t> attr8{0}, attr7{0};
  for (int64_t kb = 0; kb < k; kb += kOzakiKChunk) {
    const int64_t kc = std::min<int64_t>(kOzakiKChunk, k - kb);
    const int64_t kp = round_up(kc, 128);
    uint8_t *base = static_cast<uint8_t *>(scratch);
    int8_t *pa = reinterpret_cast<int8_t *>(base);
    int8_t *pb = pa + static_cast<int64_t>(slices) * mp * kp;
    double *sa = reinterpret_cast<double *>(
        (reinterpret_cast<uintptr_t>(pb + static_cast<int64_t>(slices) * np * kp) + 255) &
        ~static_cast<uintptr_t>(255));
    double *sb = sa + mp;
    // op(A) rows are K-contiguous unless ta; op(B) = B^T rows unless tb
    const double *a0 = ta ? A + kb * lda : A + kb;
    const double *b0 = tb ? B + kb : B + kb * ldb;
    const int at = ta ? 1 : 0, bt = tb ? 0 : 1;
    count_launch(2);
    ozaki::row_scale_kernel<<<ozaki::grid_blocks(m * 32), 256, 0, st>>>(a0, m, kc, lda, at, sa);
    ozaki::row_scale_kernel<<<ozaki::grid_blocks(n * 32), 256, 0, st>>>(b0, n, kc, ldb, bt, sb);
    const dim3 ga(static_cast<unsigned>(kp / 128), static_cast<unsigned>(mp / 32));
    const dim3 gb(static_cast<unsigned>(kp / 128), static_cast<unsigned>(np / 32));
    count_launch(2);
    if (slices == 8) {
      ozaki::operand_slice_kernel<8><<<ga, 256, 0, st>>>(a0, m, kc, lda, at, sa, pa, mp, kp);
      ozaki::operand_slice_kernel<8><<<gb, 256, 0, st>>>(b0, n, kc, ldb, bt, sb, pb, np, kp);
    } else {
      ozaki::operand_slice_kernel<7><<<ga, 256, 0, st>>>(a0, m, kc, lda, at, sa, pa, mp, kp);
      ozaki::operand_slice_kernel<7><<<gb, 256, 0, st>>>(b0, n, kc, ldb, bt, sb, pb, np, kp);
    }
    ozaki::UpdateArgs p{};
    if (!ozaki::make_operand_map(&p.tm_a, pa, kp, mp, slices, ozaki::BM) ||
        !ozaki::make_operand_map(&p.tm_b, pb, kp, np, slices, ozaki::BN))
      return MBPT_ERR_SHAPE;
    p.n = 0;
    p.j0 = 0;
    p.nb = 0;
    p.k_tiles = static_cast<int>(kp / ozaki::BKB);
    p.nmat = 1;
    p.a_row0 = p.b_row0 = 0;
    p.tiles_m = static_cast<int>(mp / ozaki::BM);
    p.tiles_n = static_cast<int>((n + ozaki::BN - 1) / ozaki::BN);
    p.P = nullptr;
    p.p_stride = 0;
    p.scale = sa;
    p.scale_b = sb;
    p.rowsq = nullptr;
    p.C = C;
    p.ldc = ldc;
    p.alpha = alpha;
    p.beta = kb == 0 ? beta : 1.0;
    p.m_rows = static_cast<int>(m);
    p.n_cols = static_cast<int>(n);
    p.sym = x.sym ? 1 : 0;
    p.H1 = x.h1;
    p.H2 = x.h1 ? x.h2 : nullptr;
    p.C2 = x.c2;
    p.err = err;
    const dim3 grid(static_cast<unsigned>(p.tiles_m * p.tiles_n), 1);
    count_launch();
    if (slices == 8) {
      auto kern = ozaki::chol_update_kernel<8, ozaki::EPI_GEMM>;
      const int smem = ozaki::Layout<8>::kSmemBytes;
      if (!allow_smem(reinterpret_cast<const void *>(kern), smem, attr8)) return MBPT_ERR_CUDA;
      kern<<<grid, 192, smem, st>>>(p);
    } else {
      auto kern = ozaki::chol_update_kernel<7, ozaki::EPI_GEMM>;
      const int smem = ozaki::Layout<7>::kSmemBytes;
      if (!allow_smem(reinterpret_cast<const void *>(kern), smem, attr7)) return MBPT_ERR_CUDA;
      kern<<<grid, 192, smem, st>>>(p);
    }
    if (cudaGetLastError() != cudaSuccess) return MBPT_ERR_CUDA;
  }
  return MBPT_OK;
}

}  // namespace mbpt
