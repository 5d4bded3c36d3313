// Shared definitions of the libmbpt_b200 kernels: status codes, bounded waits,
// BF16 split helpers. sm_100a only.
#pragma once
#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "../../include/mbpt_b200.h"

namespace mbpt {

using bf16 = __nv_bfloat16;

// A device-side wait gives up after this many nanoseconds of wall time
// (%globaltimer) and reports MBPT_ERR_TIMEOUT through the call's error word.
constexpr uint64_t kWaitLimitNs = 4000000000ull;

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// x = hi + lo with hi = bf16(x), lo = bf16(x - hi): 16 significant bits.
__device__ __forceinline__ void split_bf16(float x, bf16 &hi, bf16 &lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// x rounded to TF32 (10 explicit mantissa bits, to nearest with ties away
// from zero) as an FP32 word with the low 13 bits clear. Finite inputs only.
__device__ __forceinline__ float to_tf32(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// x = hi + lo with hi = tf32(x), lo = tf32(x - hi): 22 significant bits.
__device__ __forceinline__ void split_tf32(float x, float &hi, float &lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - hi);
}

__host__ __device__ __forceinline__ int64_t round_up(int64_t x, int64_t m) {
  return (x + m - 1) / m * m;
}

// Largest matrix extent the stand-alone GEMM entry points take (2^24): with
// every extent at most this, the padded products and their byte counts
// (below 2^52) cannot wrap in int64_t or size_t.
constexpr int64_t kMaxGemmExtent = int64_t(1) << 24;
__host__ __device__ __forceinline__ bool gemm_extents_ok(int64_t m, int64_t n, int64_t k) {
  return m >= 1 && n >= 1 && k >= 1 && m <= kMaxGemmExtent && n <= kMaxGemmExtent &&
         k <= kMaxGemmExtent;
}

// Error word written by kernels that detect a failure on the device (a wait
// that ran out). Zeroed by the host before a call, read back after it.
struct DevErr {
  int *word;
  __device__ __forceinline__ void set(int code) const {
    if (word) atomicCAS(word, 0, code);
  }
};

// Number of this library's kernels launched by the process (instrumentation).
void count_launch(int n = 1);

}  // namespace mbpt

#define MBPT_CUDA(call)                                                    \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return MBPT_ERR_CUDA;                             \
  } while (0)

#define MBPT_LAUNCH_CHECK()                                                  \
  do {                                                                       \
    cudaError_t e_ = cudaGetLastError();                                     \
    if (e_ != cudaSuccess) return MBPT_ERR_CUDA;                             \
  } while (0)
