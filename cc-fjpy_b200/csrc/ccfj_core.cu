// Host-side plumbing of the C-ABI: errors, allocator, launch counter, the
// autotuners' table.
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>

#include "ccfj_core.cuh"
#include "tune_cache.h"

namespace ccfj {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
std::mutex g_alloc_mu;
ccfj_alloc_fn g_alloc = nullptr;
ccfj_free_fn g_free = nullptr;
void* g_alloc_user = nullptr;
}  // namespace

int set_error(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

void clear_error() { g_last_error.clear(); }

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ------------------------------------------------------ autotuner table
// In-process choices of both autotuners, keyed by (tuner, class key, device
// name), backed by the file named by ccfj_set_tune_cache or, by default,
// the environment variable CCFJ_TUNE_CACHE (no file: in-process only). The
// file is read on the first lookup of each device, and every tuning result
// is written through to it.
namespace {
std::mutex g_tune_mu;
std::map<std::pair<std::string, std::string>, int> g_tunes;  // (kind + device, key) -> choice
std::map<std::string, bool> g_tune_loaded;                   // device -> read
bool g_tune_path_set = false;
std::string g_tune_path;

// The current device's name token (queried once per device ordinal).
std::string current_device_token() {
  static std::mutex mu;
  static std::map<int, std::string> names;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return tune::device_token("");
  std::lock_guard<std::mutex> lk(mu);
  auto it = names.find(dev);
  if (it != names.end()) return it->second;
  cudaDeviceProp p{};
  const std::string t =
      tune::device_token(cudaGetDeviceProperties(&p, dev) == cudaSuccess ? p.name : "");
  names[dev] = t;
  return t;
}

std::string tune_path_locked() {
  if (g_tune_path_set) return g_tune_path;
  const char* env = std::getenv("CCFJ_TUNE_CACHE");
  return env ? std::string(env) : std::string();
}

std::pair<std::string, std::string> tune_slot(const std::string& kind, const std::string& device,
                                              long long key) {
  return {kind + "|" + device, std::to_string(key)};
}

void tune_load_locked(const std::string& device) {
  if (g_tune_loaded[device]) return;
  g_tune_loaded[device] = true;
  const std::string path = tune_path_locked();
  if (path.empty()) return;
  for (const tune::Entry& e : tune::read_file(path))
    if (e.device == device) g_tunes[tune_slot(e.kind, e.device, e.key)] = e.choice;
}
}  // namespace

bool tune_lookup(const char* kind, long long key, int* choice) {
  const std::string device = current_device_token();
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_load_locked(device);
  auto it = g_tunes.find(tune_slot(kind, device, key));
  if (it == g_tunes.end()) return false;
  *choice = it->second;
  return true;
}

int tune_record(const char* kind, long long key, int choice, float ms) {
  const std::string device = current_device_token();
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_load_locked(device);
  g_tunes[tune_slot(kind, device, key)] = choice;
  const std::string path = tune_path_locked();
  if (path.empty()) return CCFJ_OK;
  tune::Entry e;
  e.device = device;
  e.kind = kind;
  e.key = key;
  e.choice = choice;
  e.ms = ms;
  if (!tune::upsert_file(path, e))
    return set_error(CCFJ_ERR_INVALID, "autotuner: cannot write the table %s", path.c_str());
  return CCFJ_OK;
}

// Scratch comes from one stream-ordered memory pool per device that keeps
// its memory between calls (release threshold = max): without it, every
// call would map its multi-GB scratch afresh from the driver.
static cudaMemPool_t library_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

void* dev_alloc(size_t bytes, cudaStream_t s) {
  if (bytes == 0) bytes = 256;
  ccfj_alloc_fn fn;
  void* user;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    fn = g_alloc;
    user = g_alloc_user;
  }
  if (fn) {
    void* p = fn(bytes, (void*)s, user);
    if (!p) set_error(CCFJ_ERR_ALLOC, "allocator hook returned NULL for %zu bytes", bytes);
    return p;
  }
  void* p = nullptr;
  // during stream capture the allocation becomes a graph memory node, which
  // the graph manages itself: take it from the default pool then
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (s) cudaStreamIsCapturing(s, &cs);
  cudaMemPool_t pool = cs == cudaStreamCaptureStatusNone ? library_pool() : nullptr;
  cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, s) : cudaMallocAsync(&p, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(CCFJ_ERR_ALLOC, "cudaMallocAsync(%zu) failed: %s", bytes, cudaGetErrorString(e));
    return nullptr;
  }
  return p;
}

void dev_free(void* p, cudaStream_t s) {
  if (!p) return;
  ccfj_free_fn fn;
  void* user;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    fn = g_free;
    user = g_alloc_user;
  }
  if (fn) {
    fn(p, (void*)s, user);
    return;
  }
  cudaFreeAsync(p, s);
}

bool allocator_hooked() {
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  return g_alloc != nullptr;
}

Scratch::~Scratch() {
  for (int i = n_ - 1; i >= 0; --i) dev_free(ptrs_[i], s_);
}

void* Scratch::get(size_t bytes) {
  if (n_ >= 32) {
    set_error(CCFJ_ERR_ALLOC, "internal: too many scratch buffers");
    return nullptr;
  }
  void* p = dev_alloc((bytes + 255) & ~size_t(255), s_);
  if (p) ptrs_[n_++] = p;
  return p;
}

}  // namespace ccfj

CCFJ_API const char* ccfj_last_error(void) { return ccfj::g_last_error.c_str(); }

CCFJ_API const char* ccfj_version(void) { return "ccfj_b200 0.1.0 (sm_100a)"; }

CCFJ_API long long ccfj_launch_count(void) {
  return ccfj::g_launches.load(std::memory_order_relaxed);
}

CCFJ_API int ccfj_set_allocator(ccfj_alloc_fn alloc, ccfj_free_fn free_fn, void* user) {
  if ((alloc == nullptr) != (free_fn == nullptr))
    return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_set_allocator: give both functions or neither");
  std::lock_guard<std::mutex> lk(ccfj::g_alloc_mu);
  ccfj::g_alloc = alloc;
  ccfj::g_free = free_fn;
  ccfj::g_alloc_user = user;
  return CCFJ_OK;
}

CCFJ_API int ccfj_host_alloc(size_t bytes, void** ptr) {
  ccfj::clear_error();
  if (!ptr) return ccfj::set_error(CCFJ_ERR_INVALID, "ccfj_host_alloc: ptr is NULL");
  *ptr = nullptr;
  const cudaError_t e = cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    return ccfj::set_error(CCFJ_ERR_ALLOC, "ccfj_host_alloc: cudaHostAlloc(%zu) failed: %s", bytes,
                           cudaGetErrorString(e));
  }
  return CCFJ_OK;
}

CCFJ_API int ccfj_host_free(void* ptr) {
  ccfj::clear_error();
  if (!ptr) return CCFJ_OK;
  const cudaError_t e = cudaFreeHost(ptr);
  if (e != cudaSuccess)
    return ccfj::set_error(CCFJ_ERR_CUDA, "ccfj_host_free: %s", cudaGetErrorString(e));
  return CCFJ_OK;
}

CCFJ_API int ccfj_set_tune_cache(const char* path) {
  ccfj::clear_error();
  std::lock_guard<std::mutex> lk(ccfj::g_tune_mu);
  ccfj::g_tune_path_set = path != nullptr;
  ccfj::g_tune_path = path ? path : "";
  ccfj::g_tune_loaded.clear();  // read the (new) table again on the next lookup
  return CCFJ_OK;
}
