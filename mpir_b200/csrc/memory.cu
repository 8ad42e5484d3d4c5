// Device memory of the engine: stream-ordered allocations from each device's
// default memory pool.
//
// cudaFree waits for the whole device; with several host threads each
// driving its own stream (the serving engine), every free would stall every
// other thread's work.  Allocations here are cudaMallocAsync on one
// allocation stream per device, made visible to all streams by a
// synchronisation of that stream alone; frees are cudaFreeAsync on it and do
// not wait.  The engine frees a buffer only once the work that used it has
// completed (its owner synchronised its streams), so the pool may hand the
// memory out again at once.  Freed memory stays in the pool (release
// threshold at its maximum); an allocation that does not fit first returns
// the pool's unused memory to the device and tries once more.
//
// The serving engine's worker threads allocate with plain cudaMalloc
// instead (set_thread_pool(false)): with eight workers holding the device
// near its capacity, pool allocations that had to grow the pool took several
// times longer than cudaMalloc (measured: 40 s against 6 s of the workers'
// time setting up new factors on a 160-request stream).  Their frees go to
// a cache of idle blocks (at most kCacheBytes) instead of cudaFree, which
// would wait for the whole device; an allocation takes the smallest cached
// block of its device that is at least its size and at most a quarter (plus
// 2 MiB) larger, else calls cudaMalloc, and one that does not fit first
// frees the cached blocks (so does a pool allocation that does not fit, and
// the serving engine when it is destroyed).  A refactorization of a pattern seen before finds
// its scratch buffers' sizes there.  MPIR_ALLOC=sync makes cudaMalloc and
// the cache the default of every thread.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "engine.hpp"

namespace mpir {

namespace {
constexpr int  kMaxDevices = 64;
std::once_flag g_once[kMaxDevices];
cudaStream_t   g_stream[kMaxDevices];

cudaStream_t alloc_stream(int d) {
  if (d < 0 || d >= kMaxDevices) throw CudaError(cudaErrorInvalidDevice, "allocation stream");
  std::call_once(g_once[d], [d] {
    cudaMemPool_t pool;
    MPIR_CUDA(cudaDeviceGetDefaultMemPool(&pool, d));
    uint64_t keep = UINT64_MAX;
    MPIR_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    MPIR_CUDA(cudaStreamCreateWithFlags(&g_stream[d], cudaStreamNonBlocking));
  });
  return g_stream[d];
}

// Makes device d current for the scope.
struct OnDevice {
  int prev = -1;
  explicit OnDevice(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~OnDevice() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

thread_local int t_pool = -1;  // -1: the process default

// Idle cudaMalloc blocks.
struct Idle {
  void    *p;
  size_t   cap;
  int      device;
  uint64_t seq;
};
constexpr size_t  kCacheBytes = size_t{24} << 30;
std::mutex        g_cache_mu;
std::vector<Idle> g_cache;
size_t            g_cache_bytes = 0;
uint64_t          g_cache_seq   = 0;

// Takes a cached block for `bytes` on device d (nullptr: none fits).
void *cache_take(size_t bytes, int d, size_t *cap) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  const size_t hi   = bytes + bytes / 4 + (size_t{2} << 20);
  size_t       best = g_cache.size();
  for (size_t i = 0; i < g_cache.size(); i++) {
    const Idle &c = g_cache[i];
    if (c.device == d && c.cap >= bytes && c.cap <= hi &&
        (best == g_cache.size() || c.cap < g_cache[best].cap))
      best = i;
  }
  if (best == g_cache.size()) return nullptr;
  void *p = g_cache[best].p;
  *cap    = g_cache[best].cap;
  g_cache_bytes -= *cap;
  g_cache[best] = g_cache.back();
  g_cache.pop_back();
  return p;
}

// Frees the cached blocks of device d (all when d < 0); the caller's device
// is current for d.
void cache_flush(int d) {
  std::vector<Idle> out;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (size_t i = 0; i < g_cache.size();) {
      if (d < 0 || g_cache[i].device == d) {
        out.push_back(g_cache[i]);
        g_cache_bytes -= g_cache[i].cap;
        g_cache[i] = g_cache.back();
        g_cache.pop_back();
      } else {
        i++;
      }
    }
  }
  for (const Idle &c : out)
    if (cudaFree(c.p) != cudaSuccess) cudaGetLastError();
}

bool use_pool() {
  static const bool pool = [] {
    const char *e = std::getenv("MPIR_ALLOC");
    return e == nullptr || std::strcmp(e, "sync") != 0;
  }();
  return t_pool < 0 ? pool : t_pool != 0;
}
}  // namespace

void set_thread_pool(bool pool) { t_pool = pool ? 1 : 0; }

void *device_alloc(size_t bytes, DevMem *m) {
  int d = 0;
  MPIR_CUDA(cudaGetDevice(&d));
  m->device = d;
  m->pooled = use_pool();
  m->cap    = bytes;
  if (!m->pooled) {
    if (void *p = cache_take(bytes, d, &m->cap)) return p;
    void       *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      cache_flush(d);
      e = cudaMalloc(&p, bytes);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(e, "cudaMalloc");
    }
    return p;
  }
  cudaStream_t s = alloc_stream(d);
  void        *p = nullptr;
  cudaError_t  e = cudaMallocAsync(&p, bytes, s);
  if (e == cudaErrorMemoryAllocation) {
    // the pool's unused memory and the cache's idle blocks go back to the
    // device, then one more try
    cudaGetLastError();
    cudaMemPool_t pool;
    MPIR_CUDA(cudaStreamSynchronize(s));
    MPIR_CUDA(cudaDeviceGetDefaultMemPool(&pool, d));
    MPIR_CUDA(cudaMemPoolTrimTo(pool, 0));
    cache_flush(d);
    e = cudaMallocAsync(&p, bytes, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw CudaError(e, "cudaMallocAsync");
  }
  MPIR_CUDA(cudaStreamSynchronize(s));  // usable from every stream from here on
  return p;
}

void device_free(void *p, const DevMem &m) {
  if (!p) return;
  OnDevice on(m.device);
  if (!m.pooled) {
    std::vector<Idle> out;  // the oldest blocks beyond the cache's size
    {
      std::lock_guard<std::mutex> lk(g_cache_mu);
      g_cache.push_back({p, m.cap, m.device, g_cache_seq++});
      g_cache_bytes += m.cap;
      while (g_cache_bytes > kCacheBytes) {
        size_t old = 0;
        for (size_t i = 1; i < g_cache.size(); i++)
          if (g_cache[i].seq < g_cache[old].seq) old = i;
        out.push_back(g_cache[old]);
        g_cache_bytes -= g_cache[old].cap;
        g_cache[old] = g_cache.back();
        g_cache.pop_back();
      }
    }
    for (const Idle &c : out) {
      OnDevice od(c.device);
      if (cudaFree(c.p) != cudaSuccess) cudaGetLastError();
    }
    return;
  }
  // Errors are ignored: a free at process exit may come after the context.
  if (cudaFreeAsync(p, alloc_stream(m.device)) != cudaSuccess) cudaGetLastError();
}

// Pinned host blocks: cudaFreeHost waits for the whole device as cudaFree
// does, so freed blocks are kept (at most kPinnedCache bytes) for the next
// request of the same size.
namespace {
constexpr size_t                          kPinnedCache = size_t{64} << 20;
std::mutex                                g_pin_mu;
std::vector<std::pair<void *, size_t>>    g_pin;
size_t                                    g_pin_bytes = 0;
}  // namespace

void *pinned_alloc(size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    for (size_t i = 0; i < g_pin.size(); i++)
      if (g_pin[i].second == bytes) {
        void *p = g_pin[i].first;
        g_pin_bytes -= bytes;
        g_pin[i] = g_pin.back();
        g_pin.pop_back();
        return p;
      }
  }
  void *p = nullptr;
  MPIR_CUDA(cudaMallocHost(&p, bytes));
  return p;
}

void pinned_free(void *p, size_t bytes) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pin_bytes + bytes <= kPinnedCache) {
      g_pin.emplace_back(p, bytes);
      g_pin_bytes += bytes;
      return;
    }
  }
  if (cudaFreeHost(p) != cudaSuccess) cudaGetLastError();
}

void device_zero(void *p, size_t bytes) {
  int d = 0;
  MPIR_CUDA(cudaGetDevice(&d));
  cudaStream_t s = alloc_stream(d);
  MPIR_CUDA(cudaMemsetAsync(p, 0, bytes, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
}

void device_cache_flush(int device) {
  OnDevice on(device);
  cache_flush(device);
}

size_t device_free_bytes(int device) {
  OnDevice on(device);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (const Idle &c : g_cache)
      if (c.device == device) free_b += c.cap;
  }
  // memory the pool holds but no buffer uses is free for the engine too
  cudaMemPool_t pool;
  uint64_t      reserved = 0, used = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
      reserved > used)
    free_b += static_cast<size_t>(reserved - used);
  cudaGetLastError();
  return free_b;
}

}  // namespace mpir
