// Split-precision tensor-core GEMM engine for sm_100a (tcgen05 + TMA + TMEM).
//
// Every product of the route's N^3 sweeps is C = A B^T with A (m x K) and
// B (n x K) both K-contiguous, each operand held as a BF16 pair x = hi + lo.
// One CTA owns a 128 x BN output tile and one or two accumulators in TMEM
// (each its own (A, B, K) problem, e.g. G_occ and G_virt of the same grid
// tile); a CTA pair (cta_group::2) owns a 256 x BN tile, 128 rows each.
// Per 64-wide K slab it issues three tcgen05.mma per 16-wide step,
// hi*hi + hi*lo + lo*hi, all into the same FP32 accumulator (the lo*lo term,
// 2^-18 relative, is dropped). Warp roles: warp 0 issues the TMA loads
// (128B swizzle, no multicast), warp 1 owns TMEM and issues the MMAs, warps
// 2-5 run the fused epilogue (Hadamard products, BF16 re-split, FP32 stores
// or the self-energy row contraction). Every mbarrier wait is bounded: on
// timeout the kernel records MBPT_ERR_TIMEOUT, drains and returns.
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace mbpt {
namespace umma {

constexpr int BM = 128;
constexpr int BK = 64;  // BF16 elements per 128-byte swizzle row
constexpr int kGroupM = 16;

enum Epi : int {
  EPI_SPLIT = 0,           // out0 = alpha * acc0, BF16 hi/lo
  EPI_F32 = 1,             // outf = alpha * acc0, FP32
  EPI_HADAMARD_SPLIT = 2,  // out0 = acc0 o acc1, BF16 hi/lo   (Pi = Go o Gv)
  EPI_SIGMA_HZ = 3,        // out0 = acc0 o Zt, out1 = acc1 o Zt, Zt read (FP32) at zt
  EPI_ROWDOT2 = 4,         // sig0[c] += sum_r xs[r,c] acc0[r,c], sig1[c] -= ... acc1
  EPI_F32_ACC = 5,         // outf += alpha * acc0, FP32 read-modify-write
  EPI_TF32_PAIR = 6,       // alpha * acc0 as a TF32 hi/lo pair at p (and transposed at t)
  EPI_F64_SYM = 7,         // outd = alpha * acc0 - shift [row == col], FP64, rows and
                           // columns below nd, mirrored (with BAND_UPPER)
};

struct EpiArgs {
  bf16 *out0_hi = nullptr, *out0_lo = nullptr, *out1_hi = nullptr, *out1_lo = nullptr;
  int64_t ld_out = 0;
  float *outf = nullptr;
  int64_t ld_outf = 0;
  float alpha = 1.f;
  const float *xs = nullptr;
  int64_t ld_xs = 0;
  double *sig0 = nullptr, *sig1 = nullptr;
  // EPI_TF32_PAIR: row-major pair p (ld_p) and, when t_hi is set, the
  // transposed pair t (element (r, c) of the tile grid at t[c * ld_t + r])
  float *p_hi = nullptr, *p_lo = nullptr, *t_hi = nullptr, *t_lo = nullptr;
  int64_t ld_p = 0, ld_t = 0;
  // EPI_F64_SYM: the nd x nd FP64 output (leading dimension ld_outd)
  double *outd = nullptr;
  int64_t ld_outd = 0;
  int nd = 0;
  double shift = 0.0;
  // EPI_SIGMA_HZ: the FP32 factor of both products, row-major (ld_zt)
  const float *zt = nullptr;
  int64_t ld_zt = 0;
};

// Structure of triangular operands, for products whose rows vanish on one
// side of the diagonal in K: each output tile then runs only the K slabs that
// can be nonzero (and, for a symmetric product, only tiles on or above the
// diagonal). A row r of A (rows = the M dimension) that is zero for k < r
// gives BAND_K_FROM_M: the tile starting at row m0 starts its K loop at m0.
enum Band : int {
  BAND_K_FROM_M = 1,  // A(r, k) = 0 for k < r
  BAND_K_FROM_N = 2,  // B(r, k) = 0 for k < r
  BAND_K_TO_M = 4,    // A(r, k) = 0 for k > r
  BAND_K_TO_N = 8,    // B(r, k) = 0 for k > r
  BAND_UPPER = 16,    // symmetric output: tiles below the diagonal are not formed
                      // (the FP32 / pair / Hadamard epilogues store each tile above
                      // the diagonal twice, the second time transposed)
};

// Grouped launch (one accumulator): independent products of one launch, each
// a block of the same A and B arrays. Coordinates are elements of those
// arrays; the Band spans apply within each product.
struct Group {
  int tile_base;       // first linear tile of this product in the launch
  int tiles_m, tiles_n;
  int a_row0, a_k0;    // origin of the product's A block (row, K)
  int b_row0, b_k0;    // origin of its B block
  int k_tiles;         // K slabs from the origin
  int64_t p_off, t_off;  // element offsets of its output (and transposed output)
  int m_valid, n_valid;  // its output rows and columns (tiles past them store nothing)
};

template <int NACC, int NGRP = 0>
struct Params {
  CUtensorMap tm[4 * NACC];  // per accumulator: A hi, A lo, B hi, B lo
  int k_tiles[NACC];
  int tiles_m, tiles_n;
  int n_valid;  // output columns to store (tiles_n * BN unless the last tile overhangs)
  int m_valid;  // output rows to store (a CTA pair's second tile may lie past them)
  int band;  // Band flags (0: dense)
  int ngroups;
  Group grp[NGRP > 0 ? NGRP : 1];
  EpiArgs epi;
  int *err;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false once kWaitLimitNs have passed without the phase flipping.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity,
                                          uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t t0 = global_ns();
  while (true) {
#pragma unroll 1
    for (int i = 0; i < 64; ++i)
      if (mbar_try_wait(b, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// ---- CTA pairs (cluster of 2, cta_group::2) ----
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// The shared::cluster address of this CTA's shared variable *p as held by CTA
// `rank` of the cluster (the same offset in that CTA's shared memory).
__device__ __forceinline__ uint32_t cluster_addr(const void *p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
  return a;
}

// Every thread of both CTAs of the cluster.
__device__ __forceinline__ void cluster_sync() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_bar) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on a barrier that the other CTA of the pair also arrives on.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t *b, uint32_t parity,
                                                  uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait_cluster(b, parity)) return true;
  const uint64_t t0 = global_ns();
  while (true) {
#pragma unroll 1
    for (int i = 0; i < 64; ++i)
      if (mbar_try_wait_cluster(b, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// A tile into this CTA's shared memory whose bytes complete on a barrier of
// either CTA of the pair (`bar` a shared::cluster address). No multicast.
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *tm, int x, int y,
                                                 uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), Blackwell descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>(1) << 16;
  d |= static_cast<uint64_t>(1024 >> 4) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(2) << 61;
  return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = m (128, or
// 256 for a CTA pair), N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, int m = 128) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

// Instruction descriptor: TF32 x TF32 -> FP32, both K-major, M = m (128, or
// 256 for a CTA pair), N = n.
__host__ __device__ constexpr uint32_t idesc_tf32(int n, int m = 128) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

// One 32-byte K step (8 TF32 or 16 BF16 elements) of the three split
// products hi*hi + hi*lo + lo*hi into accumulator d; `first` overwrites it.
template <bool TF32>
__device__ __forceinline__ void mma3(uint32_t d, uint64_t a_hi, uint64_t a_lo, uint64_t b_hi,
                                     uint64_t b_lo, uint32_t idesc, uint32_t first) {
  if constexpr (TF32) {
    mma_tf32(d, a_hi, b_hi, idesc, first ? 0u : 1u);
    mma_tf32(d, a_hi, b_lo, idesc, 1u);
    mma_tf32(d, a_lo, b_hi, idesc, 1u);
  } else {
    mma_bf16(d, a_hi, b_hi, idesc, first ? 0u : 1u);
    mma_bf16(d, a_hi, b_lo, idesc, 1u);
    mma_bf16(d, a_lo, b_hi, idesc, 1u);
  }
}

// One MMA of a CTA pair, issued by the pair's first CTA: A's rows and B's
// rows are split between the two CTAs' shared memory at the same offsets, and
// each CTA's TMEM receives its own 128 rows. No output lane is disabled.
__device__ __forceinline__ void mma_bf16_pair(uint32_t tmem_d, uint64_t da, uint64_t db,
                                              uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, "
      "{%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u),
      "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_tf32_pair(uint32_t tmem_d, uint64_t da, uint64_t db,
                                              uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, "
      "{%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u),
      "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

template <bool TF32>
__device__ __forceinline__ void mma3_pair(uint32_t d, uint64_t a_hi, uint64_t a_lo,
                                          uint64_t b_hi, uint64_t b_lo, uint32_t idesc,
                                          uint32_t first) {
  if constexpr (TF32) {
    mma_tf32_pair(d, a_hi, b_hi, idesc, first ? 0u : 1u);
    mma_tf32_pair(d, a_hi, b_lo, idesc, 1u);
    mma_tf32_pair(d, a_lo, b_hi, idesc, 1u);
  } else {
    mma_bf16_pair(d, a_hi, b_hi, idesc, first ? 0u : 1u);
    mma_bf16_pair(d, a_hi, b_lo, idesc, 1u);
    mma_bf16_pair(d, a_lo, b_hi, idesc, 1u);
  }
}

// Completion of the pair's MMAs issued so far, arriving once on the barrier
// at `bar`'s offset in both CTAs.
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(smem_u32(bar)),
      "h"(static_cast<uint16_t>(3))
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane, waited on in place.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(addr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void store_split32(bf16 *hi, bf16 *lo, const float (&v)[32]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    __align__(16) bf16 h[8];
    __align__(16) bf16 l[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) split_bf16(v[8 * q + i], h[i], l[i]);
    reinterpret_cast<uint4 *>(hi)[q] = *reinterpret_cast<const uint4 *>(h);
    reinterpret_cast<uint4 *>(lo)[q] = *reinterpret_cast<const uint4 *>(l);
  }
}

// The transposed store of store_split32: v[i] goes to hi/lo[i * ld] (base at
// the mirrored position); across the warp, lanes (consecutive rows) write
// consecutive elements of each mirrored row.
__device__ __forceinline__ void store_split32_t(bf16 *hi, bf16 *lo, int64_t ld,
                                                const float (&v)[32]) {
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    bf16 h, l;
    split_bf16(v[i], h, l);
    hi[i * ld] = h;
    lo[i * ld] = l;
  }
}

// Lane l ends with the warp sum of column l of the 32 x 32 block v (row = lane).
__device__ __forceinline__ float warp_column_sum(float (&v)[32], int lane) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int i = 0; i < s; ++i) {
      const float send = upper ? v[i] : v[i + s];
      const float keep = upper ? v[i + s] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
  return v[0];
}


// CTAS = 2: a CTA pair computes a 256 x BN tile, each CTA holding its 128
// rows of A and half of B's BN rows in a stage.
template <int NACC, int BN, bool DRAIN = false, int CTAS = 1>
struct Layout {
  static constexpr int kABytes = BM * BK * 2;
  static constexpr int kBBytes = BN / CTAS * BK * 2;
  static constexpr int kStageBytes = 2 * kABytes + 2 * kBBytes;
  static constexpr int kStages = (kStageBytes <= 64 * 1024) ? 3 : 2;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 256;
  // a drained last accumulator takes two buffers; two 256-wide accumulators
  // with a drain fit only as the drained one first, the other reusing one of
  // its buffers (kDrainFirst)
  static constexpr bool kDrainFirst = BN == 256 && NACC == 2 && DRAIN;
  static constexpr int kCols = kDrainFirst ? 2 * BN : (NACC + (DRAIN ? 1 : 0)) * BN;
  static constexpr int kTmemCols = (kCols <= 32) ? 32 : (kCols <= 64) ? 64
                                   : (kCols <= 128) ? 128 : (kCols <= 256) ? 256 : 512;
  static_assert(kCols <= 512, "accumulators exceed TMEM");
};

// TF32: operands are FP32 words holding TF32-rounded hi/lo parts (32 per
// 128-byte row, K step 8); otherwise BF16 pairs (64 per row, K step 16).
// Either way a stage holds 128-byte rows and a K step advances 32 bytes.
//
// DRAIN > 0: the tensor core's FP32 accumulation truncates, which biases a
// long K sum towards zero by about half an ulp per accumulation step (~4e-5
// relative at K = 7296 with three split products). The last accumulator is
// therefore restarted every DRAIN K slabs in one of two TMEM buffers, and the
// epilogue warps add each finished chunk into round-to-nearest FP32 sums in
// registers while the MMAs fill the other buffer.
// BN = 128: 6 warps (producer, MMA, 4 epilogue); BN = 256: 10 warps, the 8
// epilogue warps covering the TMEM lane quarters twice, 128 columns each.
//
// CTAS = 2 (launched as clusters of two; BF16 or TF32; a band's K span taken
// per pair): the CTA pair forms a 256 x BN tile with cta_group::2 MMAs issued
// by the first CTA. Each CTA loads
// its own 128 rows of A and its half of B's rows, both completing on the first
// CTA's full barrier; the commits arrive in both CTAs; the second CTA's
// epilogue warps release drained buffers on the first CTA's barrier. Per K
// slab a CTA then moves 64 KB instead of 96 KB for the same MMA work, and
// three stages fit instead of two.
template <int NACC, int BN, int EPI, bool TF32 = false, int DRAIN = 0, int NGRP = 0,
          int CTAS = 1>
__global__ void __launch_bounds__(64 + BN, 1)
    gemm_split_kernel(const __grid_constant__ Params<NACC, NGRP> p) {
  constexpr bool kPair = CTAS == 2;
  static_assert(!kPair || (BN == 256 && (NGRP == 0 ? NACC <= 2 : NACC == 1)),
                "CTA pairs: 256-wide tiles of one or two accumulators (one when grouped)");
  using L = Layout<NACC, BN, (DRAIN > 0), CTAS>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L::kStages * L::kStageBytes);
  uint64_t *empty = full + L::kStages;
  uint64_t *accum = empty + L::kStages;
  uint64_t *dfull = accum + 1;   // [2] a drained chunk is complete in buffer b
  uint64_t *dempty = dfull + 2;  // [2] the epilogue has read buffer b
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(dempty + 2);
  int *fail = reinterpret_cast<int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // rank in the pair (0 issues the MMAs); 0 without pairs
  const uint32_t rank = kPair ? cluster_rank() : 0u;
  const bool leader = rank == 0;
  // this CTA's product (grouped launches) and its origins
  int pid = kPair ? static_cast<int>(blockIdx.x >> 1) : static_cast<int>(blockIdx.x);
  int tiles_m = p.tiles_m, tiles_n = p.tiles_n;
  int a_row0 = 0, a_k0 = 0, b_row0 = 0, b_k0 = 0, grp_k_tiles = 0;
  int m_valid = p.m_valid, n_valid = p.n_valid;
  int64_t p_off = 0, t_off = 0;
  if constexpr (NGRP > 0) {
    int g = 0;
    while (g + 1 < p.ngroups && pid >= p.grp[g + 1].tile_base) ++g;
    const Group &G = p.grp[g];
    pid -= G.tile_base;
    tiles_m = G.tiles_m;
    tiles_n = G.tiles_n;
    a_row0 = G.a_row0;
    a_k0 = G.a_k0;
    b_row0 = G.b_row0;
    b_k0 = G.b_k0;
    grp_k_tiles = G.k_tiles;
    p_off = G.p_off;
    t_off = G.t_off;
    m_valid = G.m_valid;
    n_valid = G.n_valid;
  }
  // grouped raster: kGroupM row tiles sweep the column tiles together (L2
  // reuse); a pair's unit is two row tiles, so half as many units per group
  constexpr int kUnitsM = kPair ? kGroupM / 2 : kGroupM;
  const int units_m = kPair ? (tiles_m + 1) / 2 : tiles_m;
  const int per_group = kUnitsM * tiles_n;
  const int first_m = (pid / per_group) * kUnitsM;
  const int gsize = min(units_m - first_m, kUnitsM);
  const int um = first_m + (pid % per_group) % gsize;
  const int tn = (pid % per_group) / gsize;
  // the pair's first row tile; this CTA's row tile (the second CTA's may lie
  // past the last one: it computes zeros and stores nothing)
  const int tm_pair = kPair ? 2 * um : um;
  const int tm = tm_pair + static_cast<int>(rank);
  const int m0 = tm * BM, n0 = tn * BN;
  constexpr int kLast = NACC - 1;
  // the drained accumulator: the last one, or the first with kDrainFirst (its
  // chunks then go through TMEM columns [0, 2 BN) and the other accumulator
  // takes the buffer the chunk after its last would have used)
  constexpr bool kDrainFirst = L::kDrainFirst;
  constexpr int kDr = kDrainFirst ? 0 : kLast;
  // uniform across the CTA (and the pair), before any barrier or TMEM exists:
  // a symmetric product skips tiles whose last 128-column block lies below
  // the diagonal
  if ((p.band & BAND_UPPER) && (n0 + BN) / 128 - 1 < tm_pair) return;
  // K slabs [kb, ke) of accumulator j that can hold nonzeros for this tile (a
  // pair's: both CTAs run its rows' span; the slabs one CTA adds are zeros)
  constexpr int kSlab = TF32 ? 32 : BK;
  const int m_lo = tm_pair * BM, m_hi = (tm_pair + CTAS) * BM;
  auto k_span = [&](int j, int &kb, int &ke) {
    kb = 0;
    ke = NGRP > 0 ? grp_k_tiles : p.k_tiles[j];
    if (p.band & BAND_K_FROM_M) kb = max(kb, m_lo / kSlab);
    if (p.band & BAND_K_FROM_N) kb = max(kb, n0 / kSlab);
    if (p.band & BAND_K_TO_M) ke = min(ke, m_hi / kSlab);
    if (p.band & BAND_K_TO_N) ke = min(ke, (n0 + BN) / kSlab);
    ke = max(ke, kb);
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < L::kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], 1);
      // a pair's drained buffers are released by both CTAs' epilogue warps
      mbar_init(&dempty[b], CTAS * BN / 32);
    }
    *fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    if constexpr (kPair) {
      // one warp of each CTA of the pair: the same columns in both
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"(L::kTmemCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"(L::kTmemCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
  }
  tc_fence_before();
  // a pair: both CTAs' barriers exist before either CTA's loads, commits or
  // arrivals can reach them
  if constexpr (kPair)
    cluster_sync();
  else
    __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int j = 0; j < NACC && ok; ++j) {
        int kb, ke;
        k_span(j, kb, ke);
        for (int kt = kb; kt < ke; ++kt, ++it) {
          const int s = it % L::kStages;
          const uint32_t ph = (it / L::kStages) & 1;
          if (!mbar_wait(&empty[s], ph ^ 1)) { ok = false; break; }
          // a pair's stage completes on the first CTA's barrier with both
          // CTAs' bytes
          if (leader) mbar_expect_tx(&full[s], CTAS * L::kStageBytes);
          uint8_t *st = smem + s * L::kStageBytes;
          // K coordinate in elements: one 128-byte row per slab
          const int kx = kt * kSlab;
          if constexpr (kPair) {
            const uint32_t bar = cluster_addr(&full[s], 0);
            const int nb = b_row0 + n0 + static_cast<int>(rank) * (BN / 2);
            tma_load_2d_pair(st, &p.tm[4 * j + 0], a_k0 + kx, a_row0 + m0, bar);
            tma_load_2d_pair(st + L::kABytes, &p.tm[4 * j + 1], a_k0 + kx, a_row0 + m0, bar);
            tma_load_2d_pair(st + 2 * L::kABytes, &p.tm[4 * j + 2], b_k0 + kx, nb, bar);
            tma_load_2d_pair(st + 2 * L::kABytes + L::kBBytes, &p.tm[4 * j + 3], b_k0 + kx, nb,
                             bar);
          } else {
            tma_load_2d(st, &p.tm[4 * j + 0], a_k0 + kx, a_row0 + m0, &full[s]);
            tma_load_2d(st + L::kABytes, &p.tm[4 * j + 1], a_k0 + kx, a_row0 + m0, &full[s]);
            tma_load_2d(st + 2 * L::kABytes, &p.tm[4 * j + 2], b_k0 + kx, b_row0 + n0,
                        &full[s]);
            tma_load_2d(st + 2 * L::kABytes + L::kBBytes, &p.tm[4 * j + 3], b_k0 + kx,
                        b_row0 + n0, &full[s]);
          }
        }
      }
      if (!ok) {
        atomicExch(fail, 1);
        DevErr{p.err}.set(MBPT_ERR_TIMEOUT);
      }
      // drain: every load issued lands before the CTA may exit (a pair's
      // loads all complete on the first CTA's barriers, and the second CTA
      // waits for the first at the closing cluster barrier)
      const int issued = leader ? it : 0;
      for (int q = max(0, issued - L::kStages); q < issued; ++q)
        mbar_wait(&full[q % L::kStages], (q / L::kStages) & 1);
    }
    __syncwarp();
  } else if (warp == 1) {
    // a pair's MMAs are issued by its first CTA alone
    if (lane == 0 && leader) {
      constexpr uint32_t idesc =
          TF32 ? idesc_tf32(BN, CTAS * BM) : idesc_bf16(BN, CTAS * BM);
      int it = 0;
      bool ok = true;
      for (int j = 0; j < NACC && ok; ++j) {
        const bool drained = DRAIN > 0 && j == kDr;
        uint32_t d = tmem + static_cast<uint32_t>(j * BN);
        int buf = 0;
        int kb, ke;
        if constexpr (kDrainFirst) {
          if (j != kDr) {
            // the buffer of drained chunk nch, once the epilogue has read
            // chunk nch - 2 from it
            k_span(kDr, kb, ke);
            const int nch = (ke - kb + DRAIN - 1) / DRAIN;
            const uint32_t par = ((nch >> 1) & 1) ^ 1;
            if (!(kPair ? mbar_wait_cluster(&dempty[nch & 1], par)
                        : mbar_wait(&dempty[nch & 1], par))) {
              ok = false;
              break;
            }
            tc_fence_after();
            d = tmem + static_cast<uint32_t>((nch & 1) * BN);
          }
        }
        k_span(j, kb, ke);
        for (int kt = kb; kt < ke; ++kt, ++it) {
          const int q = kt - kb;  // slab index within this tile's K span
          const bool chunk_start = drained && (q % (DRAIN > 0 ? DRAIN : 1)) == 0;
          if (chunk_start) {
            const int c = q / (DRAIN > 0 ? DRAIN : 1);
            buf = c & 1;
            const uint32_t par = ((c >> 1) & 1) ^ 1;
            if (!(kPair ? mbar_wait_cluster(&dempty[buf], par) : mbar_wait(&dempty[buf], par))) {
              ok = false;
              break;
            }
            tc_fence_after();
            d = tmem + static_cast<uint32_t>((kDr + buf) * BN);
          }
          const int s = it % L::kStages;
          const uint32_t ph = (it / L::kStages) & 1;
          if (!mbar_wait(&full[s], ph) || *reinterpret_cast<volatile int *>(fail)) {
            ok = false;
            break;
          }
          tc_fence_after();
          uint8_t *st = smem + s * L::kStageBytes;
          const uint64_t a_hi = sw128_desc(smem_u32(st));
          const uint64_t a_lo = sw128_desc(smem_u32(st + L::kABytes));
          const uint64_t b_hi = sw128_desc(smem_u32(st + 2 * L::kABytes));
          const uint64_t b_lo = sw128_desc(smem_u32(st + 2 * L::kABytes + L::kBBytes));
          const bool restart = drained ? chunk_start : q == 0;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t adv = static_cast<uint64_t>(kk * 2);  // 32 bytes >> 4
            if constexpr (kPair)
              mma3_pair<TF32>(d, a_hi + adv, a_lo + adv, b_hi + adv, b_lo + adv, idesc,
                              (restart && kk == 0) ? 1u : 0u);
            else
              mma3<TF32>(d, a_hi + adv, a_lo + adv, b_hi + adv, b_lo + adv, idesc,
                         (restart && kk == 0) ? 1u : 0u);
          }
          const bool chunk_end =
              drained && ((q + 1) % (DRAIN > 0 ? DRAIN : 1) == 0 || kt + 1 == ke);
          if constexpr (kPair) {
            mma_commit_pair(&empty[s]);
            if (chunk_end) mma_commit_pair(&dfull[buf]);
          } else {
            mma_commit(&empty[s]);
            if (chunk_end) mma_commit(&dfull[buf]);
          }
        }
      }
      if (!ok) {
        atomicExch(fail, 1);
        DevErr{p.err}.set(MBPT_ERR_TIMEOUT);
      }
      if constexpr (kPair)
        mma_commit_pair(accum);
      else
        mma_commit(accum);
      mbar_wait(accum, 0);  // no MMA may still write TMEM when it is freed
    }
    __syncwarp();
  } else {
    // epilogue: a warp owns TMEM lane quarter warp % 4 (the hardware's rule)
    // and the 128 columns starting at cb
    const int sp = warp & 3;
    const int cb = ((warp - 2) >> 2) * 128;
    const uint32_t taddr = tmem + (static_cast<uint32_t>(sp * 32) << 16);
    bool ok = true;
    float acc[DRAIN > 0 ? 128 : 1];
    if constexpr (DRAIN > 0) {
#pragma unroll
      for (int i = 0; i < 128; ++i) acc[i] = 0.f;
      int kb, ke;
      k_span(kDr, kb, ke);
      const int nchunks = (ke - kb + DRAIN - 1) / DRAIN;
      for (int c = 0; c < nchunks; ++c) {
        const int b = c & 1;
        const uint32_t par = (c >> 1) & 1;
        if (!(kPair ? mbar_wait_cluster(&dfull[b], par) : mbar_wait(&dfull[b], par)) ||
            *reinterpret_cast<volatile int *>(fail)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float t[32];
          tmem_ld32(taddr + static_cast<uint32_t>((kDr + b) * BN + cb + 32 * q), t);
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[32 * q + i] += t[i];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          if constexpr (kPair)
            mbar_arrive_remote(cluster_addr(&dempty[b], 0));  // the MMAs' CTA
          else
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&dempty[b]))
                         : "memory");
        }
      }
    }
    ok = ok && (kPair ? mbar_wait_cluster(accum, 0) : mbar_wait(accum, 0)) &&
         !*reinterpret_cast<volatile int *>(fail);
    __syncwarp();
    if (!ok) {
      if (lane == 0) DevErr{p.err}.set(MBPT_ERR_TIMEOUT);
    } else {
      tc_fence_after();
      const int row = m0 + sp * 32 + lane;
      const EpiArgs &e = p.epi;
      // symmetric output, per 128-column block tb of this warp: a block below
      // the diagonal is not stored, one above it also fills its mirror
      const int tb = (n0 + cb) / 128;
      const bool upper = (p.band & BAND_UPPER) != 0;
      const bool mirror = upper && tb > tm;
      // 32 columns starting at the warp's column c of accumulator j (the
      // drained one from registers)
      int col_of[NACC];
#pragma unroll
      for (int j = 0; j < NACC; ++j) col_of[j] = j * BN;
      if constexpr (kDrainFirst) {
        int kb, ke;
        k_span(kDr, kb, ke);
        col_of[1] = (((ke - kb + DRAIN - 1) / DRAIN) & 1) * BN;
      }
      auto load = [&](int j, int c, float (&v)[32]) {
        if constexpr (DRAIN > 0) {
          if (j == kDr) {
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = acc[c + i];
            return;
          }
        }
        tmem_ld32(taddr + static_cast<uint32_t>(col_of[j] + cb + c), v);
      };
      // columns past n_valid (a 256-wide tile over a 128-multiple edge) are not
      // stored, nor the rows of a pair's second tile past m_valid
      const bool live = n0 + cb < n_valid && m0 < m_valid && !(upper && tb < tm);
#pragma unroll
      for (int c = 0; c < 128; c += 32) {
        if (!live) break;
        const int col = n0 + cb + c;
        float v0[32];
        load(0, c, v0);
        if constexpr (EPI == EPI_SPLIT) {
#pragma unroll
          for (int i = 0; i < 32; ++i) v0[i] *= e.alpha;
          store_split32(e.out0_hi + row * e.ld_out + col, e.out0_lo + row * e.ld_out + col, v0);
        } else if constexpr (EPI == EPI_F32 || EPI == EPI_F32_ACC) {
          float4 *dst = reinterpret_cast<float4 *>(e.outf + row * e.ld_outf + col);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            float4 o = make_float4(e.alpha * v0[4 * q], e.alpha * v0[4 * q + 1],
                                   e.alpha * v0[4 * q + 2], e.alpha * v0[4 * q + 3]);
            if constexpr (EPI == EPI_F32_ACC) {
              const float4 prev = dst[q];
              o.x += prev.x; o.y += prev.y; o.z += prev.z; o.w += prev.w;
            }
            dst[q] = o;
          }
          if constexpr (EPI == EPI_F32) {
            if (mirror) {
#pragma unroll
              for (int i = 0; i < 32; ++i)
                e.outf[static_cast<int64_t>(col + i) * e.ld_outf + row] = e.alpha * v0[i];
            }
          }
        } else if constexpr (EPI == EPI_F64_SYM) {
          if (row < e.nd) {
            double *dst = e.outd + static_cast<int64_t>(row) * e.ld_outd + col;
#pragma unroll
            for (int i = 0; i < 32; ++i) {
              if (col + i < e.nd) {
                const double v = static_cast<double>(e.alpha * v0[i]) -
                                 (row == col + i ? e.shift : 0.0);
                dst[i] = v;
                if (mirror) e.outd[static_cast<int64_t>(col + i) * e.ld_outd + row] = v;
              }
            }
          }
        } else if constexpr (EPI == EPI_TF32_PAIR) {
          float hi[32], lo[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const float v = e.alpha * v0[i];
            hi[i] = to_tf32(v);
            lo[i] = to_tf32(v - hi[i]);
          }
          float4 *dh = reinterpret_cast<float4 *>(e.p_hi + p_off + row * e.ld_p + col);
          float4 *dl = reinterpret_cast<float4 *>(e.p_lo + p_off + row * e.ld_p + col);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            dh[q] = make_float4(hi[4 * q], hi[4 * q + 1], hi[4 * q + 2], hi[4 * q + 3]);
            dl[q] = make_float4(lo[4 * q], lo[4 * q + 1], lo[4 * q + 2], lo[4 * q + 3]);
          }
          if (e.t_hi) {
            // column col + i of the tile is row col + i of t: the warp's 32
            // consecutive rows land on 32 consecutive floats
#pragma unroll
            for (int i = 0; i < 32; ++i) {
              e.t_hi[t_off + static_cast<int64_t>(col + i) * e.ld_t + row] = hi[i];
              e.t_lo[t_off + static_cast<int64_t>(col + i) * e.ld_t + row] = lo[i];
            }
          }
        } else if constexpr (EPI == EPI_HADAMARD_SPLIT) {
          float v1[32];
          load(1, c, v1);
#pragma unroll
          for (int i = 0; i < 32; ++i) v0[i] *= v1[i];
          store_split32(e.out0_hi + row * e.ld_out + col, e.out0_lo + row * e.ld_out + col, v0);
          if (mirror)
            store_split32_t(e.out0_hi + static_cast<int64_t>(col) * e.ld_out + row,
                            e.out0_lo + static_cast<int64_t>(col) * e.ld_out + row, e.ld_out, v0);
        } else if constexpr (EPI == EPI_SIGMA_HZ) {
          // acc0 = G_occ, acc1 = G_virt; Zt (symmetric, stored whole) from memory
          float z[32], v1[32];
          const float4 *zs = reinterpret_cast<const float4 *>(e.zt + row * e.ld_zt + col);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float4 t = zs[q];
            z[4 * q] = t.x; z[4 * q + 1] = t.y; z[4 * q + 2] = t.z; z[4 * q + 3] = t.w;
          }
#pragma unroll
          for (int i = 0; i < 32; ++i) v0[i] *= z[i];
          store_split32(e.out0_hi + row * e.ld_out + col, e.out0_lo + row * e.ld_out + col, v0);
          if (mirror)
            store_split32_t(e.out0_hi + static_cast<int64_t>(col) * e.ld_out + row,
                            e.out0_lo + static_cast<int64_t>(col) * e.ld_out + row, e.ld_out, v0);
          load(1, c, v1);
#pragma unroll
          for (int i = 0; i < 32; ++i) v1[i] *= z[i];
          store_split32(e.out1_hi + row * e.ld_out + col, e.out1_lo + row * e.ld_out + col, v1);
          if (mirror)
            store_split32_t(e.out1_hi + static_cast<int64_t>(col) * e.ld_out + row,
                            e.out1_lo + static_cast<int64_t>(col) * e.ld_out + row, e.ld_out, v1);
        } else if constexpr (EPI == EPI_ROWDOT2) {
          float v1[32], xs[32];
          load(1, c, v1);
          const float4 *src = reinterpret_cast<const float4 *>(e.xs + row * e.ld_xs + col);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float4 t = src[q];
            xs[4 * q] = t.x; xs[4 * q + 1] = t.y; xs[4 * q + 2] = t.z; xs[4 * q + 3] = t.w;
          }
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            v0[i] *= xs[i];
            v1[i] *= xs[i];
          }
          const float s0 = warp_column_sum(v0, lane);
          const float s1 = warp_column_sum(v1, lane);
          atomicAdd(e.sig0 + col + lane, static_cast<double>(s0));
          atomicAdd(e.sig1 + col + lane, -static_cast<double>(s1));
        }
      }
    }
  }

  tc_fence_before();
  // a pair: neither CTA frees its TMEM (or exits, with the other's loads or
  // arrivals still due) before both are done
  if constexpr (kPair)
    cluster_sync();
  else
    __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    if constexpr (kPair)
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                   "r"(L::kTmemCols)
                   : "memory");
    else
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                   "r"(L::kTmemCols)
                   : "memory");
  }
}

}  // namespace umma
}  // namespace mbpt
