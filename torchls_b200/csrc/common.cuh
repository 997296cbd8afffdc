// Shared device helpers for the torchls_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <utility>

#include "torchls_b200.h"

#define TLS_CHECK_LAUNCH()                                   \
  do {                                                       \
    tls_count_launch();                                      \
    cudaError_t _e = cudaGetLastError();                     \
    if (_e != cudaSuccess) return tls_set_cuda_error(_e);    \
  } while (0)

int tls_set_cuda_error(cudaError_t e);
int tls_set_error(int code, const char* msg);
void tls_count_launch();
// Adds n launches at once (a recorded graph of n of this library's kernels).
void tls_count_launches(long long n);
// This thread's launches counted so far (for the size of a recorded graph).
long long tls_launches_now();

namespace tls {

constexpr int kWarp = 32;

template <typename T>
__device__ __forceinline__ T ldg(const T* p) {
  return __ldg(p);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum within aligned groups of `lanes` lanes (power of two <= 32); fixed
// butterfly order, so the result is deterministic for a fixed `lanes`.
template <typename T>
__device__ __forceinline__ T group_sum(T v, int lanes) {
  for (int o = lanes >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block reduction of one double (fixed tree order).
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double* smem /*[BLOCK/32]*/) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = (lane < BLOCK / 32) ? smem[lane] : 0.0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

// Three block sums with one exchange: each value takes exactly the tree of
// block_sum (so the results are bitwise those of three block_sum calls), with
// two barriers instead of six. Valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ void block_sum3(double& v0, double& v1, double& v2, double (*smem)[BLOCK / 32]) {
  v0 = warp_sum(v0);
  v1 = warp_sum(v1);
  v2 = warp_sum(v2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smem[0][warp] = v0;
    smem[1][warp] = v1;
    smem[2][warp] = v2;
  }
  __syncthreads();
  if (warp == 0) {
    v0 = warp_sum((lane < BLOCK / 32) ? smem[0][lane] : 0.0);
    v1 = warp_sum((lane < BLOCK / 32) ? smem[1][lane] : 0.0);
    v2 = warp_sum((lane < BLOCK / 32) ? smem[2][lane] : 0.0);
  }
  __syncthreads();
}

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

template <typename T>
__device__ __forceinline__ double to_d(T x) {
  return static_cast<double>(x);
}

// Launch settings that depend on the device (a function's dynamic shared-memory
// attribute is set per device; occupancy and SM count are per device): one
// cache per kernel instantiation, keyed by (current device, key), thread-safe.
class DeviceGridCache {
 public:
  // *out = the cached value for (current device, key); the first call per pair
  // computes it with compute(device) under the lock (a negative result is a
  // CUDA failure and is not cached).
  template <typename F>
  int get(int key, int* out, F&& compute) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return tls_set_cuda_error(e);
    std::lock_guard<std::mutex> lock(mu_);
    auto it = values_.find({dev, key});
    if (it != values_.end()) {
      *out = it->second;
      return 0;
    }
    const int v = compute(dev);
    if (v < 0) return tls_set_cuda_error(cudaGetLastError());
    values_[{dev, key}] = v;
    *out = v;
    return 0;
  }

 private:
  std::mutex mu_;
  std::map<std::pair<int, int>, int> values_;
};

inline int grid_for(int64_t n, int block, int cap = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<int>(g);
}

}  // namespace tls
