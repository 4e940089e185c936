// hb_abi.cpp -- library identity and per-thread error reporting.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include "hb_common.cuh"
#include "hipims_b200_fused.h"

namespace hb {

static thread_local char g_err[512] = "";

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int num_sms() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return n > 0 ? n : 148;
}

}  // namespace hb

extern "C" int hb_abi_version(void) { return HB_ABI_VERSION; }

extern "C" const char *hb_last_error(void) { return hb::g_err; }

extern "C" void hb_record_sizes(size_t out[3]) {
  out[0] = sizeof(hb_ctrl);
  out[1] = sizeof(hb_instance);
  out[2] = sizeof(hb_fused_batch);
}
