// ctx.cu - context lifetime, error reporting, device scratch.
#include <cstdio>
#include <cstring>
#include "gasatt_internal.h"

namespace gasatt {

int fail(gasatt_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int cuda_fail(gasatt_ctx *ctx, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return fail(ctx, GASATT_E_CUDA, m);
}

int scratch(gasatt_ctx *ctx, size_t bytes, void **ptr) {
  if (bytes > ctx->scratch_bytes) {
    if (ctx->scratch) {
      GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      GASATT_CUDA(ctx, cudaFree(ctx->scratch));
      ctx->scratch = nullptr;
    }
    size_t nb = bytes + bytes / 4 + 4096;
    GASATT_CUDA(ctx, cudaMalloc(&ctx->scratch, nb));
    ctx->scratch_bytes = nb;
  }
  *ptr = ctx->scratch;
  return GASATT_OK;
}

}  // namespace gasatt

extern "C" {

const char *gasatt_version(void) { return "gasatt-b200 0.1 (sm_100a)"; }

int gasatt_create(gasatt_ctx **out, int device, uint64_t seed) {
  if (!out) return GASATT_E_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return GASATT_E_NODEVICE;
  }
  if (device < 0 || device >= ndev) return GASATT_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return GASATT_E_CUDA;
  gasatt_ctx *ctx = new gasatt_ctx();
  ctx->device = device;
  ctx->seed = seed;
  if (cudaMallocHost(&ctx->pinned, 4096) != cudaSuccess) {
    delete ctx;
    return GASATT_E_CUDA;
  }
  *out = ctx;
  return GASATT_OK;
}

int gasatt_destroy(gasatt_ctx *ctx) {
  if (!ctx) return GASATT_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream); else cudaDeviceSynchronize();
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  delete ctx;
  return GASATT_OK;
}

const char *gasatt_last_error(const gasatt_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int gasatt_set_stream(gasatt_ctx *ctx, void *stream) {
  if (!ctx) return GASATT_E_ARG;
  ctx->stream = (cudaStream_t)stream;
  return GASATT_OK;
}

int gasatt_synchronize(gasatt_ctx *ctx) {
  if (!ctx) return GASATT_E_ARG;
  GASATT_CUDA(ctx, cudaSetDevice(ctx->device));
  GASATT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GASATT_OK;
}

int64_t gasatt_kernel_launches(const gasatt_ctx *ctx) { return ctx ? ctx->launches : -1; }

}  // extern "C"
