/* refdrv.h - host helpers for driving the reference's own CUDA kernels with
 * MATLAB feval semantics (inputs copied to device, every non-const pointer
 * argument copied back).  TEST INFRASTRUCTURE: these drivers exist only to
 * pin the oracle against the reference kernels on a GPU. */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#define RD_CHECK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return (int)e_ + 1000; } while (0)

template <typename T>
static int rd_up(T **d, const T *h, size_t n) {
  RD_CHECK(cudaMalloc((void **)d, (n ? n : 1) * sizeof(T)));
  if (n) RD_CHECK(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}
template <typename T>
static int rd_down(T *h, const T *d, size_t n) {
  if (n) RD_CHECK(cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost));
  return 0;
}
#define RD_UP(d, h, n) do { int s_ = rd_up(&(d), (h), (n)); if (s_) return s_; } while (0)
#define RD_DOWN(h, d, n) do { int s_ = rd_down((h), (d), (n)); if (s_) return s_; } while (0)
