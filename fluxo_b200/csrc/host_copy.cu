// Large copies between pageable host memory and the device (mesh arrays, states).  A pageable
// cudaMemcpy goes through the driver's own small staging buffer with one host thread; here the host
// side moves with a parallel memcpy (OpenMP) into two page-locked 32 MiB bounce buffers of the process
// (one set per device), and the transfer of one chunk overlaps the host copy of the next.  Page-locked
// host ranges and copies below 4 MiB go directly.  Copies of the process on one device take turns.
#include <cuda_runtime.h>
#include <omp.h>

#include <cstring>
#include <mutex>

#include "host_copy.h"

namespace fluxo {
namespace {

constexpr size_t kChunk = size_t(32) << 20;
constexpr size_t kDirect = size_t(4) << 20;
constexpr int kMaxDev = 64;

struct Bounce {
  std::mutex m;
  char* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool ready = false;
};

Bounce g_bounce[kMaxDev];

bool pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

void par_memcpy(void* dst, const void* src, size_t n) {
  constexpr size_t piece = size_t(1) << 20;
  const long np = (long)((n + piece - 1) / piece);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < np; ++k) {
    const size_t o = (size_t)k * piece;
    std::memcpy((char*)dst + o, (const char*)src + o, (n - o < piece) ? n - o : piece);
  }
}

// the current device's bounce buffers (allocated at the first large copy on the device)
cudaError_t bounce(Bounce*& out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  Bounce& b = g_bounce[dev];
  out = &b;
  if (b.ready) return cudaSuccess;
  for (int k = 0; k < 2; ++k) {
    if (!b.buf[k] && (e = cudaHostAlloc((void**)&b.buf[k], kChunk, cudaHostAllocDefault)) != cudaSuccess) return e;
    if (!b.ev[k] && (e = cudaEventCreateWithFlags(&b.ev[k], cudaEventDisableTiming)) != cudaSuccess) return e;
  }
  b.ready = true;
  return cudaSuccess;
}

}  // namespace

cudaError_t copy_h2d(void* dDst, const void* hSrc, size_t bytes, cudaStream_t s) {
  if (bytes < kDirect || pinned(hSrc)) {
    cudaError_t e = cudaMemcpyAsync(dDst, hSrc, bytes, cudaMemcpyHostToDevice, s);
    return e != cudaSuccess ? e : cudaStreamSynchronize(s);
  }
  Bounce* b = nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_bounce[(dev >= 0 && dev < kMaxDev) ? dev : 0].m);
  cudaError_t e = bounce(b);
  if (e != cudaSuccess) return e;
  int k = 0;
  for (size_t o = 0; o < bytes; o += kChunk, k ^= 1) {
    const size_t n = (bytes - o < kChunk) ? bytes - o : kChunk;
    if ((e = cudaEventSynchronize(b->ev[k])) != cudaSuccess) return e;  // the slot's last transfer is done
    par_memcpy(b->buf[k], (const char*)hSrc + o, n);
    if ((e = cudaMemcpyAsync((char*)dDst + o, b->buf[k], n, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(b->ev[k], s)) != cudaSuccess) return e;
  }
  return cudaStreamSynchronize(s);
}

cudaError_t copy_d2h(void* hDst, const void* dSrc, size_t bytes, cudaStream_t s) {
  if (bytes < kDirect || pinned(hDst)) {
    cudaError_t e = cudaMemcpyAsync(hDst, dSrc, bytes, cudaMemcpyDeviceToHost, s);
    return e != cudaSuccess ? e : cudaStreamSynchronize(s);
  }
  Bounce* b = nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_bounce[(dev >= 0 && dev < kMaxDev) ? dev : 0].m);
  cudaError_t e = bounce(b);
  if (e != cudaSuccess) return e;
  // chunk c goes to slot c & 1; its host copy runs while chunk c + 1 is in transfer
  const size_t nc = (bytes + kChunk - 1) / kChunk;
  for (size_t c = 0; c <= nc; ++c) {
    if (c < nc) {
      const size_t o = c * kChunk, n = (bytes - o < kChunk) ? bytes - o : kChunk;
      const int k = (int)(c & 1);
      if ((e = cudaMemcpyAsync(b->buf[k], (const char*)dSrc + o, n, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
      if ((e = cudaEventRecord(b->ev[k], s)) != cudaSuccess) return e;
    }
    if (c > 0) {
      const size_t p = c - 1, o = p * kChunk, n = (bytes - o < kChunk) ? bytes - o : kChunk;
      const int k = (int)(p & 1);
      if ((e = cudaEventSynchronize(b->ev[k])) != cudaSuccess) return e;
      par_memcpy((char*)hDst + o, b->buf[k], n);
    }
  }
  return cudaSuccess;
}

}  // namespace fluxo
