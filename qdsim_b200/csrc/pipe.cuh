// Shared-memory streaming of row-major vector blocks (n_rows x B each) for
// the per-chunk LOBPCG kernels.  A chunk's rows are processed in sub-tiles of
// SUB rows; one sub-tile of NBLK blocks is NBLK contiguous global ranges,
// each fetched by a one-dimensional bulk copy (TMA, no multicast) that
// completes on the stage's mbarrier.  With STAGES stages, STAGES - 1
// sub-tiles are in flight while the threads work on the current one.
//
// Protocol (all threads of the CTA):
//   pipe.init(dsm, begin, end);            // barriers, prologue copies
//   for (i = 0; i < pipe.nsub; ++i) {
//     ok &= pipe.wait(i);                  // bounded wait for sub-tile i
//     ... read pipe.tile(i, a), pipe.rows(i) ...
//     pipe.release(i);                     // __syncthreads + next copy
//   }
//   pipe.finish(ok, err);                  // uniform failure handling
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "tc.cuh"

namespace qd {

constexpr uint64_t kPipeWaitNs = 1000000000ull;   // 1 s bound on every wait

template <typename TV, int B, int NBLK, int SUB, int STAGES>
struct BlockPipe {
  static constexpr int BLK = SUB * B;                 // elements of one block per stage
  // Blocks of a stage are one row (B elements, 16-byte multiple) further apart
  // than their size, so the same row of different blocks falls on different
  // shared-memory banks when a warp reads several blocks at once.
  static constexpr int BLKP = BLK + B;
  static constexpr int STAGE = NBLK * BLKP;           // elements per stage
  static constexpr size_t BAR_OFF = size_t(STAGES) * STAGE * sizeof(TV);
  static constexpr size_t BYTES = BAR_OFF + 8 * STAGES;

  TV *stage;
  uint64_t *full;
  const TV *const *src;
  int begin, end, nsub;

  // src: NBLK block base pointers (global, row-major n_rows x B).
  __device__ void init(unsigned char *dsm, const TV *const *src_, int begin_, int end_) {
    stage = reinterpret_cast<TV *>(dsm);
    full = reinterpret_cast<uint64_t *>(dsm + BAR_OFF);
    src = src_;
    begin = begin_;
    end = end_;
    nsub = (end - begin + SUB - 1) / SUB;
    if (threadIdx.x == 0) {
      for (int s = 0; s < STAGES; ++s) tc::mbar_init(&full[s], 1);
      tc::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < STAGES && i < nsub; ++i) issue(i);
  }
  __device__ int rows(int i) const { return min(SUB, end - (begin + i * SUB)); }
  __device__ int row0(int i) const { return begin + i * SUB; }
  __device__ const TV *tile(int i, int a) const { return stage + (i % STAGES) * STAGE + a * BLKP; }
  __device__ TV *tile_rw(int i, int a) { return stage + (i % STAGES) * STAGE + a * BLKP; }

  __device__ void issue(int i) {   // thread 0
    const int s = i % STAGES;
    const uint32_t bytes = uint32_t(rows(i)) * B * sizeof(TV);
    tc::mbar_arrive_expect_tx(&full[s], NBLK * bytes);
#pragma unroll
    for (int a = 0; a < NBLK; ++a)
      tc::bulk_g2s(stage + s * STAGE + a * BLKP, src[a] + size_t(row0(i)) * B, bytes, &full[s]);
  }
  __device__ bool wait(int i) {
    return tc::mbar_wait(&full[i % STAGES], (i / STAGES) & 1, kPipeWaitNs);
  }
  // Every thread is done with sub-tile i: its stage takes sub-tile i + STAGES.
  __device__ void release(int i, bool ok) {
    __syncthreads();
    if (threadIdx.x == 0 && ok && i + STAGES < nsub) issue(i + STAGES);
  }
  // Uniform failure handling; returns true when every wait succeeded.  On
  // failure thread 0 sets *err and waits (bounded) for the copies still in
  // flight so that the CTA's shared memory is not released under them.
  __device__ bool finish(bool ok, int *err) {
    if (!__syncthreads_or(!ok)) return true;
    if (threadIdx.x == 0) {
      atomicOr(err, 1);
      for (int i = nsub - STAGES > 0 ? nsub - STAGES : 0; i < nsub; ++i)
        tc::mbar_wait(&full[i % STAGES], (i / STAGES) & 1, kPipeWaitNs);
    }
    return false;
  }
};

}  // namespace qd

namespace qd {

// The same protocol for a sub-tile of NX blocks of TX followed by NW blocks of
// TW (e.g. the FP64 blocks X, HX, MX beside the FP32 search directions):
// tx(i, a) / tw(i, a) return block a of each kind in sub-tile i.  Each block
// of a stage is one row longer than its data (bank skew, as above); every
// block offset is a multiple of 16 bytes because B % 4 == 0.
template <typename TX, int NX, typename TW, int NW, int B, int SUB, int STAGES>
struct MixedPipe {
  static constexpr size_t BX = size_t(SUB + 1) * B * sizeof(TX);
  static constexpr size_t BW = size_t(SUB + 1) * B * sizeof(TW);
  static constexpr size_t STAGE = NX * BX + NW * BW;
  static constexpr size_t BAR_OFF = size_t(STAGES) * STAGE;
  static constexpr size_t BYTES = BAR_OFF + 8 * STAGES;
  static_assert(B % 4 == 0, "rows of B elements must be 16-byte multiples");

  unsigned char *stage;
  uint64_t *full;
  const void *const *src;   // NX + NW block base pointers (global, row-major n x B)
  int begin, end, nsub;

  __device__ static size_t off(int a) {
    return a < NX ? size_t(a) * BX : NX * BX + size_t(a - NX) * BW;
  }
  __device__ static size_t esz(int a) { return a < NX ? sizeof(TX) : sizeof(TW); }

  __device__ void init(unsigned char *dsm, const void *const *src_, int begin_, int end_) {
    stage = dsm;
    full = reinterpret_cast<uint64_t *>(dsm + BAR_OFF);
    src = src_;
    begin = begin_;
    end = end_;
    nsub = (end - begin + SUB - 1) / SUB;
    if (threadIdx.x == 0) {
      for (int s = 0; s < STAGES; ++s) tc::mbar_init(&full[s], 1);
      tc::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < STAGES && i < nsub; ++i) issue(i);
  }
  __device__ int rows(int i) const { return min(SUB, end - (begin + i * SUB)); }
  __device__ int row0(int i) const { return begin + i * SUB; }
  __device__ const TX *tx(int i, int a) const {
    return reinterpret_cast<const TX *>(stage + size_t(i % STAGES) * STAGE + off(a));
  }
  __device__ const TW *tw(int i, int a) const {
    return reinterpret_cast<const TW *>(stage + size_t(i % STAGES) * STAGE + off(NX + a));
  }

  __device__ void issue(int i) {   // thread 0
    const int s = i % STAGES;
    const uint32_t nr = uint32_t(rows(i));
    uint32_t total = 0;
#pragma unroll
    for (int a = 0; a < NX + NW; ++a) total += nr * B * uint32_t(esz(a));
    tc::mbar_arrive_expect_tx(&full[s], total);
#pragma unroll
    for (int a = 0; a < NX + NW; ++a) {
      const size_t e = esz(a);
      tc::bulk_g2s(stage + size_t(s) * STAGE + off(a),
                   static_cast<const unsigned char *>(src[a]) + size_t(row0(i)) * B * e,
                   nr * B * uint32_t(e), &full[s]);
    }
  }
  __device__ bool wait(int i) {
    return tc::mbar_wait(&full[i % STAGES], (i / STAGES) & 1, kPipeWaitNs);
  }
  __device__ void release(int i, bool ok) {
    __syncthreads();
    if (threadIdx.x == 0 && ok && i + STAGES < nsub) issue(i + STAGES);
  }
  __device__ bool finish(bool ok, int *err) {
    if (!__syncthreads_or(!ok)) return true;
    if (threadIdx.x == 0) {
      atomicOr(err, 1);
      for (int i = nsub - STAGES > 0 ? nsub - STAGES : 0; i < nsub; ++i)
        tc::mbar_wait(&full[i % STAGES], (i / STAGES) & 1, kPipeWaitNs);
    }
    return false;
  }
};

}  // namespace qd
