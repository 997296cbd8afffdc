// C-ABI plumbing: error reporting and version.
#include <stdio.h>
#include <string.h>

#include <atomic>

#include "common.cuh"

static thread_local char g_last_error[512] = "";
static std::atomic<long long> g_launches{0};
static thread_local long long t_launches = 0;  // this host thread's share

void tls_count_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}

void tls_count_launches(long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}

long long tls_launches_now() { return t_launches; }

extern "C" int64_t tls_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int tls_set_error(int code, const char* msg) {
  snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
  return code;
}

int tls_set_cuda_error(cudaError_t e) {
  snprintf(g_last_error, sizeof(g_last_error), "CUDA error: %s", cudaGetErrorString(e));
  return TLS_ERR_CUDA;
}

extern "C" const char* tls_last_error(void) { return g_last_error; }

extern "C" int tls_version(void) { return 1; }

extern "C" int tls_device_init(int32_t device) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return tls_set_cuda_error(e);
  return TLS_OK;
}
