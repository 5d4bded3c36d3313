// mbpt_gemm_split_static: the split-precision GEMM with its scratch in a
// fixed device array of this library, for callers that cannot allocate
// device memory themselves.
//
// Some hosts own every byte of device memory through their own allocator (a
// framework's caching pool, a fixed pre-partitioned budget) and cannot hand
// this library a workspace, nor let it call cudaMalloc. This entry point
// needs neither: its scratch (the BF16 hi/lo copies of A and B and the padded
// FP32 product) lives in g_scratch below, a file-scope __device__ array that
// every GPU loading the library holds until the process exits.
//
// In host code the name g_scratch is only a host-side stand-in, not a device
// address; its device address is looked up once per device with
// cudaGetSymbolAddress while that device is current, checked, cached, and
// passed to the kernels.
#include <mutex>

#include "internal.h"

namespace mbpt {
namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;  // 32 MiB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void *g_addr[kMaxDevices] = {nullptr};

// Device address of g_scratch on the current device (looked up on the first
// call per device), or nullptr with the CUDA status in *rc.
void *scratch_address(cudaError_t *rc) {
  int dev = -1;
  *rc = cudaGetDevice(&dev);
  if (*rc != cudaSuccess) return nullptr;
  if (dev < 0 || dev >= kMaxDevices) {
    *rc = cudaErrorInvalidDevice;
    return nullptr;
  }
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    *rc = cudaGetSymbolAddress(&p, g_scratch);
    if (*rc != cudaSuccess) return nullptr;
    g_addr[dev] = p;
  }
  return g_addr[dev];
}

size_t aligned(size_t b) { return (b + 1023) & ~static_cast<size_t>(1023); }

}  // namespace
}  // namespace mbpt

using namespace mbpt;

extern "C" {

size_t mbpt_gemm_split_static_capacity(void) { return kScratchBytes; }

int mbpt_gemm_split_static(const double *A, const double *B, int64_t m, int64_t n, int64_t k,
                           double alpha, float *C, int64_t ldc, int *err, void *stream) {
  if (m < 1 || n < 1 || k < 1 || ldc < n) return MBPT_ERR_SHAPE;
  // extents past 2^24 could make the byte counts below wrap; no such
  // product fits the array anyway
  if (!gemm_extents_ok(m, n, k)) return MBPT_ERR_WORKSPACE;
  const int64_t mp = round_up(m, 128), np = round_up(n, 128), kp = round_up(k, 64);
  const size_t a_bytes = aligned(sizeof(bf16) * mp * kp);
  const size_t b_bytes = aligned(sizeof(bf16) * np * kp);
  const size_t c_bytes = aligned(sizeof(float) * mp * np);
  if (2 * a_bytes + 2 * b_bytes + c_bytes > kScratchBytes) return MBPT_ERR_WORKSPACE;
  cudaError_t rc;
  uint8_t *base = static_cast<uint8_t *>(scratch_address(&rc));
  if (!base) return MBPT_ERR_CUDA;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  bf16 *a_hi = reinterpret_cast<bf16 *>(base);
  bf16 *a_lo = reinterpret_cast<bf16 *>(base + a_bytes);
  bf16 *b_hi = reinterpret_cast<bf16 *>(base + 2 * a_bytes);
  bf16 *b_lo = reinterpret_cast<bf16 *>(base + 2 * a_bytes + b_bytes);
  float *c = reinterpret_cast<float *>(base + 2 * a_bytes + 2 * b_bytes);
  // every scratch byte the product reads is written here first (the padding
  // as zeros), so nothing left by an earlier call is read
  launch_split_pad<double>(A, m, k, k, 1.f, a_hi, a_lo, kp, mp, kp, false, st);
  launch_split_pad<double>(B, n, k, k, 1.f, b_hi, b_lo, kp, np, kp, false, st);
  SplitMat Am{a_hi, a_lo, mp, kp, kp}, Bm{b_hi, b_lo, np, kp, kp};
  umma::EpiArgs e;
  e.outf = c;
  e.ld_outf = np;
  e.alpha = static_cast<float>(alpha);
  int s = gemm_split(umma::EPI_F32, 1, &Am, &Bm, mp, np, e, err, st);
  if (s) return s;
  if (cudaMemcpy2DAsync(C, sizeof(float) * ldc, c, sizeof(float) * np, sizeof(float) * n, m,
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MBPT_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

}  // extern "C"
