// Shared definitions for the SWD B200 kernels and the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/swd.h"

namespace swd {

// Thread-local last error string (returned by swd_last_error()).
void set_error(const char* fmt, ...);

#define SWD_CUDA(...)                                                            \
  do {                                                                           \
    cudaError_t e_ = (__VA_ARGS__);                                              \
    if (e_ != cudaSuccess) {                                                     \
      ::swd::set_error("%s:%d %s: %s", __FILE__, __LINE__, #__VA_ARGS__,         \
                       cudaGetErrorString(e_));                                  \
      return SWD_ERR_CUDA;                                                       \
    }                                                                            \
  } while (0)

#define SWD_TRY(...)                    \
  do {                                  \
    int rc_ = (__VA_ARGS__);            \
    if (rc_ != SWD_OK) return rc_;      \
  } while (0)

#define SWD_CHECK(cond, ...)                                  \
  do {                                                        \
    if (!(cond)) {                                            \
      ::swd::set_error(__VA_ARGS__);                          \
      return SWD_ERR_INVALID;                                 \
    }                                                         \
  } while (0)

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Owning device buffer (no copy; move only).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  int alloc(size_t n) {
    release();
    if (n == 0) return SWD_OK;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      set_error("cudaMalloc(%zu bytes) failed: %s", n, cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? SWD_ERR_OOM : SWD_ERR_CUDA;
    }
    bytes = n;
    return SWD_OK;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Offsets of several scratch arrays inside one allocation, each on a 256-byte boundary, so that
// a call needing many arrays makes one cudaMalloc and one cudaFree (each cudaFree synchronises
// the device).  add(n) reserves n bytes and returns their offset; add(0) reserves nothing.
struct SlabPlan {
  size_t bytes = 0;
  size_t add(size_t n) {
    const size_t o = bytes;
    bytes += (n + 255) / 256 * 256;
    return o;
  }
  template <typename T> static T* at(const DevBuf& b, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(b.p) + off);
  }
};

// n bytes at offset off of a slab, with DevBuf's accessors; it owns nothing (NULL when n is 0).
struct DevView {
  void* p = nullptr;
  size_t bytes = 0;
  DevView() = default;
  DevView(const DevBuf& b, size_t off, size_t n) : p(n ? static_cast<char*>(b.p) + off : nullptr), bytes(n) {}
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace swd
