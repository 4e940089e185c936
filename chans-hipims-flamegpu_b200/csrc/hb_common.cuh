// hb_common.cuh -- shared host/device helpers of libhipims_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "hipims_b200.h"

namespace hb {

constexpr double kHSmall = 1.0e-6;  // h_small of every reference kernel
constexpr double kG = 9.81;         // g of every reference kernel

// Thread-local last-error message (hb_abi.cpp).
int set_error(int code, const char *fmt, ...);

inline int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(HB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return HB_OK;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Blocks of `threads` covering n items (at least one block, like GET_BLOCKS
// of HC/gpu.cuh:11-21).
inline unsigned blocks_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return (unsigned)(b < 1 ? 1 : b);
}

int num_sms();

}  // namespace hb
