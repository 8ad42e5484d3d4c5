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
// The serving engine's worker threads allocate with plain cudaMalloc /
// cudaFree instead (set_thread_pool(false)): with eight workers holding the
// device near its capacity, pool allocations that had to grow the pool took
// several times longer than cudaMalloc (measured: 40 s against 6 s of the
// workers' time setting up new factors on a 160-request stream).
// MPIR_ALLOC=sync makes cudaMalloc / cudaFree the default of every thread.
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

bool use_pool() {
  static const bool pool = [] {
    const char *e = std::getenv("MPIR_ALLOC");
    return e == nullptr || std::strcmp(e, "sync") != 0;
  }();
  return t_pool < 0 ? pool : t_pool != 0;
}
}  // namespace

void set_thread_pool(bool pool) { t_pool = pool ? 1 : 0; }

void *device_alloc(size_t bytes, int *device, bool *pooled) {
  int d = 0;
  MPIR_CUDA(cudaGetDevice(&d));
  *device = d;
  *pooled = use_pool();
  if (!*pooled) {
    void *p = nullptr;
    MPIR_CUDA(cudaMalloc(&p, bytes));
    return p;
  }
  cudaStream_t s = alloc_stream(d);
  void        *p = nullptr;
  cudaError_t  e = cudaMallocAsync(&p, bytes, s);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    cudaMemPool_t pool;
    MPIR_CUDA(cudaStreamSynchronize(s));
    MPIR_CUDA(cudaDeviceGetDefaultMemPool(&pool, d));
    MPIR_CUDA(cudaMemPoolTrimTo(pool, 0));
    e = cudaMallocAsync(&p, bytes, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw CudaError(e, "cudaMallocAsync");
  }
  MPIR_CUDA(cudaStreamSynchronize(s));  // usable from every stream from here on
  return p;
}

void device_free(void *p, int device, bool pooled) {
  if (!p) return;
  OnDevice on(device);
  // Errors are ignored: a free at process exit may come after the context.
  const cudaError_t e = pooled ? cudaFreeAsync(p, alloc_stream(device)) : cudaFree(p);
  if (e != cudaSuccess) cudaGetLastError();
}

size_t device_free_bytes(int device) {
  OnDevice on(device);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    return 0;
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
