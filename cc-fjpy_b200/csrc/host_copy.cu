// Large copies between pageable host memory and the device.
//
// A result copied into pageable host memory normally goes through the
// driver's own staging at the speed of one host thread, and a fresh numpy
// array adds a first-touch page fault per page on top. Here a large result
// is split into contiguous slices, one per host thread; each thread streams
// its slice through two pinned staging buffers on a stream of its own
// (double buffering: the next chunk's transfer runs while the thread copies
// the previous one out), so that the transfers, the page faults and the host
// copies of all threads overlap. The float -> double form converts while it
// copies out (MWFJ returns doubles, src/ccfj-gpu.pyx:306). Large inputs from
// pageable memory come in the same way, the other way round.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "ccfj_core.cuh"

namespace ccfj {

namespace {

constexpr size_t kDirectBytes = (size_t)16 << 20;   // smaller results: one plain copy
constexpr size_t kDirectBytesIn = (size_t)8 << 20;  // smaller inputs: one plain copy
constexpr size_t kStageBytes = (size_t)4 << 20;    // source bytes per staging buffer
constexpr int kMaxCopyThreads = 16;

// Pinned staging buffers, two per thread, kept for the process once made.
// One staged copy at a time uses them; a call that finds them in use takes
// the unstaged route.
struct StagePool {
  std::mutex m;
  bool busy = false;
  std::vector<void*> bufs;
};
StagePool g_stage;

bool host_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // pageable memory on older drivers reports an error: clear it
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

void copy_out(void* dst, const void* src, size_t n, int kind) {
  if (kind == 0) {
    std::memcpy(dst, src, n);
    return;
  }
  double* d = static_cast<double*>(dst);
  const float* s = static_cast<const float*>(src);
  for (size_t i = 0; i < n; ++i) d[i] = (double)s[i];
}

// Unstaged: plain copy (kind 0), or through a pageable buffer of one chunk
// at a time (kind 1).
int copy_plain(void* dst, const void* dsrc, size_t n, int kind, cudaStream_t s) {
  if (kind == 0) {
    CCFJ_CUDA_TRY(cudaMemcpyAsync(dst, dsrc, n, cudaMemcpyDeviceToHost, s));
    CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
    return CCFJ_OK;
  }
  const size_t chunk = std::min(n, kStageBytes / sizeof(float));
  std::vector<float> tmp(chunk);
  for (size_t off = 0; off < n; off += chunk) {
    const size_t len = std::min(chunk, n - off);
    CCFJ_CUDA_TRY(cudaMemcpyAsync(tmp.data(), static_cast<const float*>(dsrc) + off,
                                  len * sizeof(float), cudaMemcpyDeviceToHost, s));
    CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
    copy_out(static_cast<double*>(dst) + off, tmp.data(), len, 1);
  }
  return CCFJ_OK;
}

// One thread's slice [lo, hi) (elements) through its two staging buffers.
void copy_slice(int dev, const char* src, char* dst, size_t lo, size_t hi, size_t in_elem,
                size_t out_elem, int kind, cudaEvent_t ready, void* buf0, void* buf1,
                std::atomic<int>* cuda_err) {
  cudaError_t e = cudaSetDevice(dev);
  cudaStream_t st = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  void* buf[2] = {buf0, buf1};
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ready, 0);  // after the producing kernels
  const size_t chunk = kStageBytes / in_elem;
  const size_t nchunks = (hi - lo + chunk - 1) / chunk;
  auto issue = [&](size_t j) {
    const size_t off = lo + j * chunk, len = std::min(chunk, hi - off);
    cudaError_t r = cudaMemcpyAsync(buf[j & 1], src + off * in_elem, len * in_elem,
                                    cudaMemcpyDeviceToHost, st);
    if (r == cudaSuccess) r = cudaEventRecord(ev[j & 1], st);
    return r;
  };
  for (size_t j = 0; e == cudaSuccess && j < nchunks && j < 2; ++j) e = issue(j);
  for (size_t j = 0; e == cudaSuccess && j < nchunks; ++j) {
    e = cudaEventSynchronize(ev[j & 1]);
    if (e != cudaSuccess) break;
    const size_t off = lo + j * chunk, len = std::min(chunk, hi - off);
    copy_out(dst + off * out_elem, buf[j & 1], len, kind);
    if (j + 2 < nchunks) e = issue(j + 2);
  }
  // nothing may still write into the staging buffers when they go back
  if (st) {
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    cudaStreamDestroy(st);
  }
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  if (e != cudaSuccess) cuda_err->store((int)e);
}

// One thread's slice [lo, hi) (bytes) of a host-to-device copy through its
// two staging buffers: the host copy of chunk j + 1 into one buffer runs
// while chunk j transfers from the other.
void copy_slice_h2d(int dev, const char* src, char* ddst, size_t lo, size_t hi, cudaEvent_t ready,
                    void* buf0, void* buf1, std::atomic<int>* cuda_err) {
  cudaError_t e = cudaSetDevice(dev);
  cudaStream_t st = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  void* buf[2] = {buf0, buf1};
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ready, 0);  // after the destination exists
  const size_t nchunks = (hi - lo + kStageBytes - 1) / kStageBytes;
  for (size_t j = 0; e == cudaSuccess && j < nchunks; ++j) {
    const size_t off = lo + j * kStageBytes, len = std::min(kStageBytes, hi - off);
    if (j >= 2) e = cudaEventSynchronize(ev[j & 1]);  // this buffer's last transfer is done
    if (e != cudaSuccess) break;
    std::memcpy(buf[j & 1], src + off, len);
    e = cudaMemcpyAsync(ddst + off, buf[j & 1], len, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[j & 1], st);
  }
  if (st) {
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    cudaStreamDestroy(st);
  }
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  if (e != cudaSuccess) cuda_err->store((int)e);
}

// Up to `want` threads' staging buffers (two each), made on first use; 0
// when another copy holds them or none can be had.
int acquire_stage(int want) {
  std::lock_guard<std::mutex> lk(g_stage.m);
  if (g_stage.busy) return 0;
  while ((int)g_stage.bufs.size() < 2 * want) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, kStageBytes, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    g_stage.bufs.push_back(p);
  }
  const int n = std::min(want, (int)g_stage.bufs.size() / 2);
  g_stage.busy = n >= 1;
  return n;
}

void release_stage() {
  std::lock_guard<std::mutex> lk(g_stage.m);
  g_stage.busy = false;
}

int threads_for(size_t bytes) {
  int n = (int)std::min<size_t>(kMaxCopyThreads, (bytes + kStageBytes - 1) / kStageBytes);
  const unsigned hw = std::thread::hardware_concurrency();
  if (hw > 0) n = std::min(n, (int)hw);
  return std::max(n, 1);
}

}  // namespace

int copy_from_host(void* ddst, const void* src, size_t n, cudaStream_t s) {
  if (n == 0) return CCFJ_OK;
  if (n < kDirectBytesIn || host_pinned(src)) {
    CCFJ_CUDA_TRY(cudaMemcpyAsync(ddst, src, n, cudaMemcpyHostToDevice, s));
    return CCFJ_OK;
  }
  const int nthreads = acquire_stage(threads_for(n));
  if (nthreads < 1) {
    CCFJ_CUDA_TRY(cudaMemcpyAsync(ddst, src, n, cudaMemcpyHostToDevice, s));
    return CCFJ_OK;
  }
  int dev = 0;
  cudaEvent_t ready = nullptr;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ready, s);
  std::atomic<int> cuda_err{0};
  if (e == cudaSuccess) {
    const size_t per = ((n + nthreads - 1) / nthreads + kStageBytes - 1) / kStageBytes * kStageBytes;
    std::vector<std::thread> pool;
    const char* from = static_cast<const char*>(src);
    char* to = static_cast<char*>(ddst);
    for (int t = 0; t < nthreads; ++t) {
      const size_t lo = std::min(n, (size_t)t * per), hi = std::min(n, lo + per);
      if (lo >= hi) break;
      try {
        pool.emplace_back(copy_slice_h2d, dev, from, to, lo, hi, ready, g_stage.bufs[2 * t],
                          g_stage.bufs[2 * t + 1], &cuda_err);
      } catch (...) {  // no thread to be had: this slice on the calling thread
        copy_slice_h2d(dev, from, to, lo, hi, ready, g_stage.bufs[2 * t], g_stage.bufs[2 * t + 1],
                       &cuda_err);
      }
    }
    for (std::thread& th : pool) th.join();
  }
  if (ready) cudaEventDestroy(ready);
  release_stage();
  if (e != cudaSuccess)
    return set_error(CCFJ_ERR_CUDA, "copy of the input to the device: %s", cudaGetErrorString(e));
  if (cuda_err.load() != 0)
    return set_error(CCFJ_ERR_CUDA, "copy of the input to the device: %s",
                     cudaGetErrorString((cudaError_t)cuda_err.load()));
  return CCFJ_OK;
}

int copy_to_host(void* dst, const void* dsrc, size_t n, int kind, cudaStream_t s) {
  const size_t in_elem = kind == 1 ? sizeof(float) : 1;
  const size_t out_elem = kind == 1 ? sizeof(double) : 1;
  const size_t in_bytes = n * in_elem;
  if (n == 0) {
    CCFJ_CUDA_TRY(cudaStreamSynchronize(s));
    return CCFJ_OK;
  }
  if (in_bytes < kDirectBytes || (kind == 0 && host_pinned(dst)))
    return copy_plain(dst, dsrc, n, kind, s);

  const int nthreads = acquire_stage(threads_for(in_bytes));
  if (nthreads < 1) return copy_plain(dst, dsrc, n, kind, s);
  int dev = 0;
  cudaEvent_t ready = nullptr;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ready, s);
  std::atomic<int> cuda_err{0};
  if (e == cudaSuccess) {
    // slices aligned to whole chunks, so that every chunk but the last is full
    const size_t chunk = kStageBytes / in_elem;
    const size_t per = ((n + nthreads - 1) / nthreads + chunk - 1) / chunk * chunk;
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) {
      const size_t lo = std::min(n, (size_t)t * per), hi = std::min(n, lo + per);
      if (lo >= hi) break;
      const char* src = static_cast<const char*>(dsrc);
      char* out = static_cast<char*>(dst);
      try {
        pool.emplace_back(copy_slice, dev, src, out, lo, hi, in_elem, out_elem, kind, ready,
                          g_stage.bufs[2 * t], g_stage.bufs[2 * t + 1], &cuda_err);
      } catch (...) {  // no thread to be had: this slice on the calling thread
        copy_slice(dev, src, out, lo, hi, in_elem, out_elem, kind, ready, g_stage.bufs[2 * t],
                   g_stage.bufs[2 * t + 1], &cuda_err);
      }
    }
    for (std::thread& th : pool) th.join();
  }
  if (ready) cudaEventDestroy(ready);
  release_stage();
  if (e != cudaSuccess)
    return set_error(CCFJ_ERR_CUDA, "copy of the result to the host: %s", cudaGetErrorString(e));
  if (cuda_err.load() != 0)
    return set_error(CCFJ_ERR_CUDA, "copy of the result to the host: %s",
                     cudaGetErrorString((cudaError_t)cuda_err.load()));
  return CCFJ_OK;
}

}  // namespace ccfj
