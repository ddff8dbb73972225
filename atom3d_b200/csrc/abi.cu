// Error reporting and version of the C ABI.
#include <stdio.h>
#include <string.h>

#include "a3d_common.cuh"

static thread_local char g_last_error[512] = "";

void a3d_set_error(const char* msg, const char* file, int line) {
  const char* base = strrchr(file, '/');
  snprintf(g_last_error, sizeof(g_last_error), "%s (%s:%d)", msg, base ? base + 1 : file, line);
}

extern "C" const char* a3d_last_error(void) { return g_last_error; }

extern "C" const char* a3d_version(void) { return "atom3d_b200 0.1.0 sm_100a"; }

namespace a3d {
int num_sms() {
  static int cached[kMaxDevices] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
  if (cached[dev] == 0) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 148;
    cached[dev] = sms;
  }
  return cached[dev];
}

__global__ void iota_u32_kernel(uint32_t* out, int64_t n) {
  pdl_wait();
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (uint32_t)i;
}
}  // namespace a3d
