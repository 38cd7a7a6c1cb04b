// Host helpers shared by the C ABI's translation units: status records and owned device buffers.
#pragma once

#include <cstdio>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fieldcraft_chol.h"

namespace fc {
namespace host {

inline void set_status(fc_status *st, int code, int64_t column = -1, int64_t entries = 0, int64_t limit = 0,
                       const std::string &msg = std::string()) {
  if (!st) return;
  st->code = code;
  st->reserved = 0;
  st->column = column;
  st->entries = entries;
  st->limit = limit;
  std::snprintf(st->message, sizeof(st->message), "%s", msg.c_str());
}

// A device allocation owned by a handle.
struct DeviceBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DeviceBuf() = default;
  DeviceBuf(const DeviceBuf &) = delete;
  DeviceBuf &operator=(const DeviceBuf &) = delete;
  ~DeviceBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t alloc(size_t b) {
    release();
    if (b == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      return e;
    }
    bytes = b;
    return cudaSuccess;
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

template <class T>
cudaError_t upload(DeviceBuf &buf, const std::vector<T> &host, cudaStream_t st) {
  cudaError_t e = buf.alloc(sizeof(T) * host.size());
  if (e != cudaSuccess || host.empty()) return e;
  return cudaMemcpyAsync(buf.p, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice, st);
}

}  // namespace host
}  // namespace fc
