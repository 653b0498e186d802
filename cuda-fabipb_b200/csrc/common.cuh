// common.cuh -- shared helpers of the B200 FABIPB library: error reporting,
// device buffers, and the constants every kernel needs.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdint.h>
#include <string>
#include <vector>

namespace fb {

// 1/(4*pi) with the rounding of the reference's `1.0/(4*M_PI)` (gkGlobal.c)
constexpr double kFourPiI = 1.0 / (4.0 * 3.14159265358979323846);
constexpr double kOneThird = 0.33333333333333333333333333;

// Highest Taylor order the device kernels are instantiated for.
constexpr int kMaxOrder = 8;

__host__ __device__ inline int nmom(int p) { return ((p + 1) * (p + 2) * (p + 3)) / 6; }
__host__ __device__ constexpr int nmom_c(int p) { return ((p + 1) * (p + 2) * (p + 3)) / 6; }

void set_error(const char *fmt, ...);
const char *get_error();

// Stage timing, the counterpart of the reference's -B=1 stage report: with
// FABIPB_B200_TRACE set in the environment every mark() synchronises the
// stream and prints "[fabipb_b200] scope.stage ms" to stderr; unset, mark()
// does nothing and nothing is synchronised.
bool trace_enabled();
struct StageTimer {
  const char *scope;
  cudaStream_t stream;
  bool on;
  double t;
  StageTimer(const char *sc, cudaStream_t s);
  void mark(const char *stage);
};

// Throws nothing: CUDA failures are turned into a recorded message and a
// false return so every C entry point can report 0.
#define FB_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      ::fb::set_error("%s failed at %s:%d: %s", #call, __FILE__, __LINE__,         \
                      cudaGetErrorString(e_));                                     \
      return false;                                                                \
    }                                                                              \
  } while (0)

#define FB_CHECK(cond, ...)          \
  do {                               \
    if (!(cond)) {                   \
      ::fb::set_error(__VA_ARGS__);  \
      return false;                  \
    }                                \
  } while (0)

// Device allocations owned by a context (or a set-up step), freed together
// in reverse order.  They come from the device's default memory pool, which
// is told once per device to keep freed memory (release threshold: no limit):
// contexts made and dropped in turn, and the set-up steps' temporaries, reuse
// memory that is already mapped instead of mapping it anew each time.
// Allocation is complete when alloc returns (usable from any stream);
// release waits for the device first, as cudaFree does.
bool pool_keep_memory();
struct DevArena {
  std::vector<void *> ptrs;
  size_t bytes = 0;
  bool alloc(void **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 16;
    if (!pool_keep_memory()) return false;
    cudaError_t e = cudaMallocAsync(p, n, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
      set_error("device allocation of %.3f MiB failed: %s", n / 1048576.0, cudaGetErrorString(e));
      *p = nullptr;
      return false;
    }
    ptrs.push_back(*p);
    bytes += n;
    return true;
  }
  template <typename T>
  bool alloc_n(T **p, size_t count) {
    return alloc(reinterpret_cast<void **>(p), count * sizeof(T));
  }
  template <typename T>
  bool upload(T **p, const std::vector<T> &h, cudaStream_t s) {
    if (!alloc_n(p, h.size())) return false;
    if (!h.empty()) {
      cudaError_t e = cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) {
        set_error("cudaMemcpyAsync upload failed: %s", cudaGetErrorString(e));
        return false;
      }
    }
    return true;
  }
  void release() {
    if (ptrs.empty()) return;
    cudaDeviceSynchronize();   // nothing in flight still uses the memory
    for (size_t i = ptrs.size(); i-- > 0;) cudaFreeAsync(ptrs[i], 0);
    cudaStreamSynchronize(0);
    ptrs.clear();
    bytes = 0;
  }
};

inline unsigned ceil_div(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace fb
