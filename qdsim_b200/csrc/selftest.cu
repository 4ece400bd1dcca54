// Diagnostic of the library's device-side failure path: the bounded mbarrier
// wait that every bulk-copy pipeline in this library uses (tc::mbar_wait),
// run on a barrier that nothing completes, so that it expires.  The kernel
// then takes the same exit as a production kernel whose wait expired: it
// records the error in a status word, waits (bounded) for its own bulk copy
// still in flight, and returns.  Nothing traps, faults or spins without a
// bound; the context stays usable and the host reads the status.
#include <cuda_runtime.h>
#include <algorithm>
#include "common.h"
#include "tc.cuh"

namespace {

constexpr int kCopyBytes = 256;
constexpr uint64_t kDrainLimitNs = 1000000000ull;   // bound on the drain wait

__global__ void bounded_wait_selftest_kernel(uint64_t limit_ns, const int4 *src, int with_copy,
                                             int32_t *status) {
  __shared__ __align__(16) int4 buf[kCopyBytes / 16];
  __shared__ __align__(8) uint64_t never, copied;
  if (threadIdx.x == 0) {
    qd::tc::mbar_init(&never, 1);    // one arrival expected; none is ever made
    qd::tc::mbar_init(&copied, 1);
    qd::tc::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && with_copy) {
    qd::tc::mbar_arrive_expect_tx(&copied, kCopyBytes);
    qd::tc::bulk_g2s(buf, src, kCopyBytes, &copied);
  }
  const bool ok = qd::tc::mbar_wait(&never, 0, limit_ns);
  if (!__syncthreads_or(!ok)) return;          // cannot happen: nothing arrives
  if (threadIdx.x == 0) {
    atomicOr(status, 1);
    if (with_copy) {
      // drain this CTA's own copy before its shared memory is released
      if (!qd::tc::mbar_wait(&copied, 0, kDrainLimitNs)) atomicOr(status, 2);
      else if (buf[0].x != src[0].x) atomicOr(status, 4);
    }
  }
}

}  // namespace

extern "C" int qd_bounded_wait_selftest(int64_t limit_ns, const void *d_src, int with_copy,
                                        int32_t *d_status, int32_t *h_status, void *stream) {
  if (!d_status || !h_status || limit_ns < 0) return QD_ERR_INVALID;
  if (with_copy && (!d_src || (reinterpret_cast<uintptr_t>(d_src) & 15))) return QD_ERR_INVALID;
  // at most 2 s, so the diagnostic never holds the GPU for long
  const uint64_t lim = uint64_t(std::min<int64_t>(limit_ns, 2000000000ll));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  QD_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int32_t), s));
  bounded_wait_selftest_kernel<<<1, 64, 0, s>>>(lim, static_cast<const int4 *>(d_src),
                                                with_copy ? 1 : 0, d_status);
  QD_CHECK_LAUNCH();
  QD_CUDA_TRY(cudaMemcpyAsync(h_status, d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  return (*h_status & 1) ? QD_ERR_TIMEOUT : QD_OK;
}
