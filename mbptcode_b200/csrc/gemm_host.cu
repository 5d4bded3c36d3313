// Host side of the tcgen05 split GEMM engine: TMA tensor maps and launches.
#include <cudaTypedefs.h>
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <vector>

#include <algorithm>

#include "internal.h"

namespace mbpt {
bool timing_begin(cudaStream_t st, cudaEvent_t *a, cudaEvent_t *b);
void timing_end(cudaStream_t st, int epi, cudaEvent_t a, cudaEvent_t b);

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void *p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// The dynamic shared-memory opt-in of a kernel, once per device (the
// attribute belongs to the function on the current device).
bool allow_smem(const void *kern, int bytes, std::atomic<uint64_t> &done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  const uint64_t bit = dev < 64 ? (uint64_t{1} << dev) : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return true;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
      cudaSuccess)
    return false;
  done.fetch_or(bit, std::memory_order_release);
  return true;
}

namespace {

// rows x cols matrix (cols contiguous) of BF16 or FP32 (TF32) words, boxes of
// one 128-byte row (64 BF16 / 32 FP32 columns) x box_rows, 128-byte swizzle.
bool make_tmap(CUtensorMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld,
               int box_rows, bool tf32) {
  auto fn = encode_fn();
  if (!fn) return false;
  const int64_t esz = tf32 ? 4 : 2;
  const int64_t bk = 128 / esz;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld * esz) % 16 || cols % bk) return false;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * esz)};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(bk), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m, tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16,
                  2, const_cast<void *>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// CTAS = 2: clusters of two CTAs per 256 x BN tile (cta_group::2); K-band
// spans per pair.
template <int NACC, int BN, int EPI, bool TF32, int DRAIN, int CTAS = 1>
int launch(const SplitMat *A, const SplitMat *B, int64_t m_rows, int64_t n_rows,
           const umma::EpiArgs &e, int *err, cudaStream_t st, int band = 0) {
  using L = umma::Layout<NACC, BN, (DRAIN > 0), CTAS>;
  // the last column tile may overhang a multiple of 128 (BN = 256): its
  // B rows read as zeros and its dead columns are not stored
  if (m_rows % umma::BM || n_rows % 128 || m_rows <= 0 || n_rows <= 0) return MBPT_ERR_SHAPE;
  const int64_t bk = TF32 ? 32 : 64;
  umma::Params<NACC> p;
  for (int j = 0; j < NACC; ++j) {
    if (A[j].cols != B[j].cols || A[j].cols <= 0 || A[j].rows < m_rows || B[j].rows < n_rows ||
        A[j].tf32 != TF32 || B[j].tf32 != TF32)
      return MBPT_ERR_SHAPE;
    if (!make_tmap(&p.tm[4 * j + 0], A[j].hi, A[j].rows, A[j].cols, A[j].ld, umma::BM, TF32) ||
        !make_tmap(&p.tm[4 * j + 1], A[j].lo, A[j].rows, A[j].cols, A[j].ld, umma::BM, TF32) ||
        !make_tmap(&p.tm[4 * j + 2], B[j].hi, B[j].rows, B[j].cols, B[j].ld, BN / CTAS,
                   TF32) ||
        !make_tmap(&p.tm[4 * j + 3], B[j].lo, B[j].rows, B[j].cols, B[j].ld, BN / CTAS, TF32))
      return MBPT_ERR_SHAPE;
    p.k_tiles[j] = static_cast<int>(A[j].cols / bk);
  }
  p.tiles_m = static_cast<int>(m_rows / umma::BM);
  p.tiles_n = static_cast<int>((n_rows + BN - 1) / BN);
  p.n_valid = static_cast<int>(n_rows);
  p.m_valid = static_cast<int>(m_rows);
  p.band = band;
  p.ngroups = 0;
  p.epi = e;
  p.err = err;
  auto kern = umma::gemm_split_kernel<NACC, BN, EPI, TF32, DRAIN, 0, CTAS>;
  static std::atomic<uint64_t> attr_set{0};  // one bit per device
  if (!allow_smem(reinterpret_cast<const void *>(kern), L::kSmemBytes, attr_set))
    return MBPT_ERR_CUDA;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  const bool timed = timing_begin(st, &ev0, &ev1);
  count_launch();
  if constexpr (CTAS == 2) {
    // a pair per 256-row unit; an odd last row tile pairs with rows past the
    // end (zero operands, nothing stored)
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(static_cast<unsigned>(2 * ((p.tiles_m + 1) / 2) * p.tiles_n));
    cfg.blockDim = dim3(64 + BN);
    cfg.dynamicSmemBytes = L::kSmemBytes;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t rc = cudaLaunchKernelEx(&cfg, kern, p);
    if (timed) timing_end(st, EPI, ev0, ev1);
    return rc == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
  } else {
    kern<<<p.tiles_m * p.tiles_n, 64 + BN, L::kSmemBytes, st>>>(p);
    if (timed) timing_end(st, EPI, ev0, ev1);
    return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
  }
}

// The 256-wide BF16 products run as CTA pairs unless MBPT_ENGINE_PAIRS=0.
bool engine_pairs() {
  const char *v = std::getenv("MBPT_ENGINE_PAIRS");
  return !(v && v[0] == '0');
}

constexpr int kMaxGroups = 32;

// One grouped launch of up to kMaxGroups single-accumulator TF32 products:
// 128 x 128 tiles one CTA each, or (CTAS = 2) 256 x 256 tiles on CTA pairs,
// whose overhang past a product's 128-multiple edges reads neighbouring rows
// and stores nothing (each group's m_valid / n_valid).
template <int EPI, int DRAIN, int BN = 128, int CTAS = 1>
int launch_grouped(const SplitMat &A, const SplitMat &B, const GemmGroup *g, int ng,
                   const umma::EpiArgs &e, int *err, cudaStream_t st, int band) {
  using L = umma::Layout<1, BN, (DRAIN > 0), CTAS>;
  if (!A.tf32 || !B.tf32 || ng < 1 || ng > kMaxGroups) return MBPT_ERR_SHAPE;
  umma::Params<1, kMaxGroups> p;
  if (!make_tmap(&p.tm[0], A.hi, A.rows, A.cols, A.ld, umma::BM, true) ||
      !make_tmap(&p.tm[1], A.lo, A.rows, A.cols, A.ld, umma::BM, true) ||
      !make_tmap(&p.tm[2], B.hi, B.rows, B.cols, B.ld, BN / CTAS, true) ||
      !make_tmap(&p.tm[3], B.lo, B.rows, B.cols, B.ld, BN / CTAS, true))
    return MBPT_ERR_SHAPE;
  int tiles = 0;
  for (int i = 0; i < ng; ++i) {
    const GemmGroup &q = g[i];
    const int64_t kp = (q.k + 31) / 32 * 32;
    // every block inside its array, K origins on 32-element slabs
    if (q.m_rows <= 0 || q.n_rows <= 0 || q.m_rows % umma::BM || q.n_rows % 128 || q.k <= 0 ||
        q.a_k0 % 32 || q.b_k0 % 32 || q.a_row0 < 0 || q.b_row0 < 0 ||
        q.a_row0 + q.m_rows > A.rows || q.b_row0 + q.n_rows > B.rows ||
        q.a_k0 + kp > A.cols || q.b_k0 + kp > B.cols)
      return MBPT_ERR_SHAPE;
    umma::Group &G = p.grp[i];
    G.tile_base = tiles;
    G.tiles_m = static_cast<int>(q.m_rows / umma::BM);
    G.tiles_n = static_cast<int>((q.n_rows + BN - 1) / BN);
    G.m_valid = static_cast<int>(q.m_rows);
    G.n_valid = static_cast<int>(q.n_rows);
    G.a_row0 = static_cast<int>(q.a_row0);
    G.a_k0 = static_cast<int>(q.a_k0);
    G.b_row0 = static_cast<int>(q.b_row0);
    G.b_k0 = static_cast<int>(q.b_k0);
    G.k_tiles = static_cast<int>(kp / 32);
    G.p_off = q.p_off;
    G.t_off = q.t_off;
    // launch units: tiles, or pairs of row tiles
    tiles += (CTAS == 2 ? (G.tiles_m + 1) / 2 : G.tiles_m) * G.tiles_n;
  }
  p.ngroups = ng;
  p.k_tiles[0] = 0;
  p.tiles_m = p.tiles_n = 0;
  p.n_valid = 1 << 30;
  p.m_valid = 1 << 30;
  p.band = band;
  p.epi = e;
  p.err = err;
  auto kern = umma::gemm_split_kernel<1, BN, EPI, true, DRAIN, kMaxGroups, CTAS>;
  static std::atomic<uint64_t> attr_set{0};  // one bit per device
  if (!allow_smem(reinterpret_cast<const void *>(kern), L::kSmemBytes, attr_set))
    return MBPT_ERR_CUDA;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  const bool timed = timing_begin(st, &ev0, &ev1);
  count_launch();
  cudaError_t rc;
  if constexpr (CTAS == 2) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(static_cast<unsigned>(2 * tiles));
    cfg.blockDim = dim3(64 + BN);
    cfg.dynamicSmemBytes = L::kSmemBytes;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    rc = cudaLaunchKernelEx(&cfg, kern, p);
  } else {
    kern<<<tiles, 64 + BN, L::kSmemBytes, st>>>(p);
    rc = cudaGetLastError();
  }
  if (timed) timing_end(st, EPI, ev0, ev1);
  return rc == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

}  // namespace

int gemm_split_grouped(int epi, const SplitMat &A, const SplitMat &B, const GemmGroup *groups,
                       int ngroups, const umma::EpiArgs &e, int *err, cudaStream_t st,
                       int band) {
  constexpr int kDrain = 2;
  for (int first = 0; first < ngroups; first += kMaxGroups) {
    const int ng = std::min(kMaxGroups, ngroups - first);
    int rc = MBPT_ERR_UNSUPPORTED;
    if (epi == umma::EPI_TF32_PAIR)
      rc = engine_pairs()
               ? launch_grouped<umma::EPI_TF32_PAIR, kDrain, 256, 2>(A, B, groups + first, ng, e,
                                                                     err, st, band)
               : launch_grouped<umma::EPI_TF32_PAIR, kDrain>(A, B, groups + first, ng, e, err,
                                                             st, band);
    if (rc) return rc;
  }
  return MBPT_OK;
}

// ---- self-test of the engine's bounded barrier wait ----
namespace {
// One thread waits, with the engine's wait routine, on a shared-memory
// mbarrier of arrival count 1 that it first completes itself (arrive) or
// that nothing completes; a wait that gives up writes MBPT_ERR_TIMEOUT.
__global__ void wait_selftest_kernel(int arrive, uint64_t limit_ns, int *err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    umma::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (arrive)
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_u32(&bar))
                   : "memory");
    if (!umma::mbar_wait(&bar, 0, limit_ns)) DevErr{err}.set(MBPT_ERR_TIMEOUT);
  }
}
}  // namespace

int wait_selftest(int arrive, int64_t limit_us, int *err, cudaStream_t st) {
  if (limit_us < 1 || limit_us > 1000000) return MBPT_ERR_SHAPE;
  count_launch();
  wait_selftest_kernel<<<1, 32, 0, st>>>(arrive, static_cast<uint64_t>(limit_us) * 1000u, err);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

// ---- optional per-launch timing of the engine (CUDA events on the stream) ----
namespace {
struct Timing {
  std::mutex mu;
  bool on = false;
  bool tagged = true;  // also time launches made under a timing_tag
  struct Rec {
    int epi;
    cudaEvent_t a, b;
  };
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;  // events of drained records, reused
  double total_ms[8] = {0};
  long long launches[8] = {0};
  cudaEvent_t take() {
    cudaEvent_t e = nullptr;
    if (!pool.empty()) {
      e = pool.back();
      pool.pop_back();
    } else {
      cudaEventCreate(&e);
    }
    return e;
  }
};
Timing &timing() {
  static Timing t;
  return t;
}
thread_local int g_timing_tag = -1;
}  // namespace

void timing_tag(int tag) { g_timing_tag = tag; }

bool timing_begin(cudaStream_t st, cudaEvent_t *a, cudaEvent_t *b) {
  Timing &t = timing();
  std::lock_guard<std::mutex> g(t.mu);
  if (!t.on || (!t.tagged && g_timing_tag >= 0)) return false;
  *a = t.take();
  *b = t.take();
  cudaEventRecord(*a, st);
  return true;
}

void timing_end(cudaStream_t st, int epi, cudaEvent_t a, cudaEvent_t b) {
  Timing &t = timing();
  cudaEventRecord(b, st);
  std::lock_guard<std::mutex> g(t.mu);
  t.pending.push_back({g_timing_tag >= 0 ? g_timing_tag : epi, a, b});
}

int gemm_timing(int enable, double *total_ms, long long *launches) {
  Timing &t = timing();
  std::lock_guard<std::mutex> g(t.mu);
  for (auto &r : t.pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.b) != cudaSuccess) return MBPT_ERR_CUDA;
    cudaEventElapsedTime(&ms, r.a, r.b);
    t.total_ms[r.epi & 7] += ms;
    t.launches[r.epi & 7] += 1;
    t.pool.push_back(r.a);
    t.pool.push_back(r.b);
  }
  t.pending.clear();
  if (total_ms && launches) {
    for (int i = 0; i < 8; ++i) {
      total_ms[i] = t.total_ms[i];
      launches[i] = t.launches[i];
      t.total_ms[i] = 0;
      t.launches[i] = 0;
    }
  }
  t.on = enable != 0;
  t.tagged = enable != 2;
  return MBPT_OK;
}

int gemm_split(int epi, int nacc, const SplitMat *A, const SplitMat *B, int64_t m_rows,
               int64_t n_rows, const umma::EpiArgs &e, int *err, cudaStream_t st, int band) {
  using namespace umma;
  // K slabs per drained chunk of the last accumulator: 24 accumulation steps
  // (~1e-6 relative truncation bias, against ~4e-5 for an undrained K = 7296)
  constexpr int kDrain = 2;
  const bool tf = nacc > 0 && A[0].tf32;
  if (band == BAND_UPPER && !(tf && nacc == 1)) {
    // symmetric products of full K: the upper tiles, mirrored by the epilogue
    if (m_rows != n_rows) return MBPT_ERR_SHAPE;
    if (tf && nacc == 2 && epi == EPI_HADAMARD_SPLIT) {
      if (engine_pairs()) {
        // 256-wide pairs: the drained (long, second) product goes first, the
        // other reuses one of its TMEM buffers; the Hadamard is symmetric
        const SplitMat A2[2] = {A[1], A[0]}, B2[2] = {B[1], B[0]};
        return launch<2, 256, EPI_HADAMARD_SPLIT, true, kDrain, 2>(A2, B2, m_rows, n_rows, e,
                                                                   err, st, band);
      }
      return launch<2, 128, EPI_HADAMARD_SPLIT, true, kDrain>(A, B, m_rows, n_rows, e, err, st,
                                                              band);
    }
    if (!tf && nacc == 1 && epi == EPI_F32)
      return engine_pairs()
                 ? launch<1, 256, EPI_F32, false, kDrain, 2>(A, B, m_rows, n_rows, e, err, st,
                                                            band)
                 : launch<1, 256, EPI_F32, false, kDrain>(A, B, m_rows, n_rows, e, err, st,
                                                         band);
    // the two G products of Sigma's H (short K: not drained) against a stored Zt
    if (!tf && nacc == 2 && epi == EPI_SIGMA_HZ)
      return engine_pairs()
                 ? launch<2, 256, EPI_SIGMA_HZ, false, 0, 2>(A, B, m_rows, n_rows, e, err, st,
                                                            band)
                 : launch<2, 256, EPI_SIGMA_HZ, false, 0>(A, B, m_rows, n_rows, e, err, st,
                                                         band);
    if (!tf && nacc == 1 && epi == EPI_F64_SYM)
      return engine_pairs()
                 ? launch<1, 256, EPI_F64_SYM, false, kDrain, 2>(A, B, m_rows, n_rows, e, err,
                                                                st, band)
                 : launch<1, 256, EPI_F64_SYM, false, kDrain>(A, B, m_rows, n_rows, e, err, st,
                                                             band);
    return MBPT_ERR_UNSUPPORTED;
  }
  if (band) {
    // triangular K spans: the single drained FP32-store TF32 product only (its
    // spans are never empty for the operand shapes the flags describe)
    if (!tf || nacc != 1 || (epi != EPI_F32 && epi != EPI_TF32_PAIR && epi != EPI_F64_SYM))
      return MBPT_ERR_UNSUPPORTED;
    if ((band & BAND_UPPER) && m_rows != n_rows) return MBPT_ERR_SHAPE;
    if (epi == EPI_TF32_PAIR)
      return launch<1, 128, EPI_TF32_PAIR, true, kDrain>(A, B, m_rows, n_rows, e, err, st,
                                                         band);
    // the symmetric FP64 store (W = L^-T L^-1): 128 x 256 tiles, which halve
    // the A reads through shared memory for the three TF32 products
    if (epi == EPI_F64_SYM && (band & BAND_UPPER))
      return engine_pairs()
                 ? launch<1, 256, EPI_F64_SYM, true, kDrain, 2>(A, B, m_rows, n_rows, e, err,
                                                               st, band)
                 : launch<1, 256, EPI_F64_SYM, true, kDrain>(A, B, m_rows, n_rows, e, err, st,
                                                            band);
    if (epi == EPI_F64_SYM)
      return launch<1, 128, EPI_F64_SYM, true, kDrain>(A, B, m_rows, n_rows, e, err, st, band);
    return launch<1, 128, EPI_F32, true, kDrain>(A, B, m_rows, n_rows, e, err, st, band);
  }
  if (tf) {
    if (nacc == 2 && epi == EPI_HADAMARD_SPLIT)
      return launch<2, 128, EPI_HADAMARD_SPLIT, true, kDrain>(A, B, m_rows, n_rows, e, err, st);
    if (nacc == 1 && epi == EPI_F32)
      return launch<1, 128, EPI_F32, true, kDrain>(A, B, m_rows, n_rows, e, err, st);
    if (nacc == 1 && epi == EPI_TF32_PAIR)
      return launch<1, 128, EPI_TF32_PAIR, true, kDrain>(A, B, m_rows, n_rows, e, err, st);
    return MBPT_ERR_UNSUPPORTED;
  }
  // the non-symmetric N^3 products: 128 x 256 tiles (a quarter fewer operand
  // bytes per flop through the shared-memory ring than 128 x 128)
  if (nacc == 1 && epi == EPI_SPLIT)
    return engine_pairs()
               ? launch<1, 256, EPI_SPLIT, false, kDrain, 2>(A, B, m_rows, n_rows, e, err, st)
               : launch<1, 256, EPI_SPLIT, false, kDrain>(A, B, m_rows, n_rows, e, err, st);
  if (nacc == 1 && epi == EPI_F32)
    return launch<1, 128, EPI_F32, false, kDrain>(A, B, m_rows, n_rows, e, err, st);
  if (nacc == 1 && epi == EPI_F32_ACC)
    return launch<1, 128, EPI_F32_ACC, false, kDrain>(A, B, m_rows, n_rows, e, err, st);
  if (nacc == 2 && epi == EPI_HADAMARD_SPLIT)
    return launch<2, 128, EPI_HADAMARD_SPLIT, false, kDrain>(A, B, m_rows, n_rows, e, err, st);
  // the row contraction: two undrained accumulators, 256-wide on CTA pairs
  if (nacc == 2 && epi == EPI_ROWDOT2)
    return engine_pairs()
               ? launch<2, 256, EPI_ROWDOT2, false, 0, 2>(A, B, m_rows, n_rows, e, err, st)
               : launch<2, 128, EPI_ROWDOT2, false, 0>(A, B, m_rows, n_rows, e, err, st);
  return MBPT_ERR_UNSUPPORTED;
}

}  // namespace mbpt
