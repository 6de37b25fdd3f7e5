// Shared host-side plumbing of the ccfj_b200 C-ABI: status codes, the
// per-thread error message, device-memory allocation through an injectable
// allocator, and launch checks. No entry point ever exits the process or
// resets the device (the reference's checkCudaErrors does both,
// include/cuda_helper.h:73-84); every failure becomes a status code plus a
// message readable through ccfj_last_error().
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/ccfj_b200.h"

namespace ccfj {

// Records a message for ccfj_last_error() and returns the status unchanged.
int set_error(int status, const char* fmt, ...);
void clear_error();

// Device memory goes through these so that a caller (and the failure tests)
// can substitute an allocator. With no hook installed, stream-ordered
// cudaMallocAsync / cudaFreeAsync are used.
void* dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);
// True when ccfj_set_allocator installed a caller allocator.
bool allocator_hooked();

// A scope that frees everything it allocated, in reverse order, on the
// stream it was created with.
class Scratch {
 public:
  explicit Scratch(cudaStream_t s) : s_(s) {}
  ~Scratch();
  // Returns nullptr on failure (and records the error).
  void* get(size_t bytes);
  template <typename T>
  T* get_n(size_t n) {
    return static_cast<T*>(get(n * sizeof(T)));
  }

 private:
  cudaStream_t s_;
  void* ptrs_[32] = {};
  int n_ = 0;
};

#define CCFJ_CUDA_TRY(expr)                                                                  \
  do {                                                                                       \
    cudaError_t e__ = (expr);                                                                \
    if (e__ != cudaSuccess) {                                                                \
      cudaGetLastError(); /* a non-sticky error must not fail a later launch check */       \
      return ::ccfj::set_error(CCFJ_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,                \
                               cudaGetErrorString(e__), __FILE__, __LINE__);                 \
    }                                                                                        \
  } while (0)

#define CCFJ_LAUNCH_CHECK(name)                                                              \
  do {                                                                                       \
    cudaError_t e__ = cudaGetLastError();                                                    \
    if (e__ != cudaSuccess)                                                                  \
      return ::ccfj::set_error(CCFJ_ERR_CUDA, "launch of %s failed: %s", name,               \
                               cudaGetErrorString(e__));                                     \
  } while (0)

#define CCFJ_REQUIRE(cond, ...)                                                              \
  do {                                                                                       \
    if (!(cond)) return ::ccfj::set_error(CCFJ_ERR_INVALID, __VA_ARGS__);                    \
  } while (0)

// Copies a result from device memory to host memory `dst` (pageable or
// pinned) after the work queued on `s`, and waits for it. kind 0: `n`
// bytes; kind 1: `n` floats stored as doubles. Large copies run through
// pinned staging buffers on several host threads (host_copy.cu).
int copy_to_host(void* dst, const void* dsrc, size_t n, int kind, cudaStream_t s);
// Copies n bytes of input from host memory to device memory ddst, ordered
// after the work queued on s. A large copy from pageable memory runs
// through the same staging on several host threads and is complete on
// return; other copies are queued on s (cudaMemcpyAsync).
int copy_from_host(void* ddst, const void* src, size_t n, cudaStream_t s);

// Optional event timer around the main transform kernel (ccfj_profile_enable).
void prof_begin(cudaStream_t s);
void prof_end(cudaStream_t s);

// The autotuners' table: the recorded choice of tuner `kind` ("fj",
// "batch") for a problem class on the current device, and a new record
// (written through to the persistent table when one is configured; the
// status reports a failed write).
bool tune_lookup(const char* kind, long long key, int* choice);
int tune_record(const char* kind, long long key, int choice, float ms);

// Counts kernel launches issued by this library (per process); the benchmark
// reads it to report how many of its own kernels a step launched.
void count_launch(int n = 1);

inline unsigned div_up(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace ccfj
