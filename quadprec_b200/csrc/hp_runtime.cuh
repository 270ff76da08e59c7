// Host runtime shared by the CUDA translation units: status codes, error
// reporting, the library stream and stream-ordered device allocations.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/hyperprec_gpu.h"

namespace hp {

// Thread-local text of the last failure (read through hp_last_error()).
void set_error(const char* fmt, ...);
const char* last_error();

// The library's own non-blocking stream for the host-pointer entry points
// (one per device, created on first use).
cudaStream_t library_stream();
// Two more per-device streams for host<->device copies that overlap the
// library stream's kernels (0: host to device, 1: device to host).
cudaStream_t library_copy_stream(int which);

// Stream-ordered device memory from the device's default pool. The pool is
// configured once to keep freed blocks cached, so repeated calls of the same
// size do not return memory to the driver.
void* dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);

// Device-side status word (one per device) used by kernels that spin or
// detect data errors. Kernels only ever OR bits into it; it stays set until
// consume_device_status() reads and clears it. consume_device_status
// synchronises s and returns HP_ERR_TIMEOUT when a bounded wait gave up.
uint32_t* device_status(cudaStream_t s);
int consume_device_status(cudaStream_t s);
enum : uint32_t {
  DEV_STATUS_TIMEOUT = 1u,      // a bounded wait gave up
  DEV_STATUS_NOT_SPD = 2u,      // a Cholesky pivot was <= 0
  DEV_STATUS_NONFINITE = 4u,    // a non-finite input was met where unsupported
};

// Optional phase timing (hp_profile_enable / hp_profile_read): drivers call
// profile_mark(stream, "phase") at phase boundaries; when profiling is off
// this is a no-op. Used by bench.py to time the dominant kernel on its own
// stream with CUDA events.
void profile_mark(cudaStream_t s, const char* name);
bool profiling_on();

struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t st) : s(st) { p = bytes ? dev_alloc(bytes, st) : nullptr; }
  ~DevBuf() {
    if (p) dev_free(p, s);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

inline bool mul_overflows(size_t a, size_t b, size_t* out) {
  if (a != 0 && b > SIZE_MAX / a) return true;
  *out = a * b;
  return false;
}

}  // namespace hp

#define HP_CUDA_TRY(expr)                                                                    \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      hp::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e));     \
      return HP_ERR_CUDA;                                                                    \
    }                                                                                        \
  } while (0)

#define HP_LAUNCH_CHECK()                                                                    \
  do {                                                                                       \
    cudaError_t _e = cudaGetLastError();                                                     \
    if (_e != cudaSuccess) {                                                                 \
      hp::set_error("%s:%d: kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(_e)); \
      return HP_ERR_CUDA;                                                                    \
    }                                                                                        \
  } while (0)

#define HP_TRY(expr)          \
  do {                        \
    int _rc = (expr);         \
    if (_rc != HP_OK) return _rc; \
  } while (0)
