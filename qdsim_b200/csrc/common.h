// Shared host/device helpers for libqdsim_b200 (status codes, launch checks).
#pragma once
#include <cstdint>
#include <cstddef>
#include <atomic>
#include "../../include/qdsim_b200.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace qd {

// counts kernels launched by this library (reported by qd_kernel_launch_count)
extern std::atomic<uint64_t> g_launches;

// Optional per-kernel-kind timing with CUDA events (qd_prof_*).  Disabled by
// default; when enabled every instrumented launch records an event pair on its
// own stream, resolved by qd_prof_read.
enum ProfKind { PK_SPMM = 0, PK_GRAM, PK_RR, PK_UPDATE, PK_ASSEMBLE, PK_PCG, PK_ADJOINT, PK_PRECOND,
                PK_ORTHO, PK_OTHER, PK_COUNT };
#ifdef __CUDACC__
bool prof_enabled();
void prof_begin(int kind, cudaStream_t s);
void prof_end(int kind, cudaStream_t s);
#endif

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Bump allocator over a caller-provided workspace.
struct Arena {
  char *base;
  size_t size;
  size_t used;
  Arena(void *p, size_t n) : base(static_cast<char *>(p)), size(n), used(0) {}
  template <typename T>
  T *take(size_t count) {
    size_t off = align_up(used, 256);
    size_t bytes = align_up(count * sizeof(T), 256);
    if (base == nullptr) {  // size query mode
      used = off + bytes;
      return nullptr;
    }
    if (off + bytes > size) return nullptr;
    used = off + bytes;
    return reinterpret_cast<T *>(base + off);
  }
};

}  // namespace qd

#ifdef __CUDACC__
#define QD_CUDA_TRY(expr)                                  \
  do {                                                     \
    cudaError_t _e = (expr);                               \
    if (_e != cudaSuccess) return QD_ERR_CUDA;             \
  } while (0)
#define QD_LAUNCHED() qd::g_launches.fetch_add(1, std::memory_order_relaxed)
#define QD_CHECK_LAUNCH()                                  \
  do {                                                     \
    QD_LAUNCHED();                                         \
    cudaError_t _e = cudaGetLastError();                   \
    if (_e != cudaSuccess) return QD_ERR_CUDA;             \
  } while (0)
#endif
