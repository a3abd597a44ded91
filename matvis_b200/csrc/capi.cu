// Library-level C ABI: version, error messages, device information.
#include <mutex>

#include "common.cuh"

namespace mvb {

std::string &last_error() {
  static thread_local std::string msg;
  return msg;
}

// SM count of the current device, cached per device ordinal.
int num_sms() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

}  // namespace mvb

extern "C" int mvb_version(void) { return 1; }

extern "C" const char *mvb_last_error(void) { return mvb::last_error().c_str(); }

extern "C" int mvb_device_info(int *sm_count, int *cc_major, int *cc_minor) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return mvb::fail(MVB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  int a = 0, b = 0, c = 0;
  cudaDeviceGetAttribute(&a, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&b, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&c, cudaDevAttrComputeCapabilityMinor, dev);
  if (sm_count) *sm_count = a;
  if (cc_major) *cc_major = b;
  if (cc_minor) *cc_minor = c;
  return MVB_OK;
}
