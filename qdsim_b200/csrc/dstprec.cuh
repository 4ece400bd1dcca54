// Fast-sine-transform preconditioner for LOBPCG on structured rectangular
// meshes (no reference counterpart; the reference's eigensolves are
// unpreconditioned ARPACK / dense solves).
//
// For a dot whose reduced DOFs are the interior points of an nx x ny lattice
// (row-major), T = (cx Kx + cy Ky + shift I)^-1 where Kx, Ky are the 1-D
// second-difference matrices: the P1 stiffness of the lattice, spectrally
// equivalent to the P1/P2/P3 stiffness of the finite-element mesh, plus a
// shift that makes it positive definite.  DST-I diagonalises Kx and Ky, so
//   T R = Sx Sy (Lambda^-1 o (Sy Sx R)),   S symmetric orthonormal, S = S^-1,
// i.e. two transform-GEMMs along x and two along y per application, run for
// all dots and all B columns at once on the tensor cores (tcgen05, BF16
// operands, FP32 accumulation in TMEM).  A preconditioner only steers the
// search directions (the Rayleigh-Ritz step is exact), and a relative
// perturbation of T of the size of the BF16 rounding leaves the condition
// number of T A, and with it the iteration count, unchanged.
//
// Vector data of one dot is a 3-D array [slow][k][b] or [k][fast] seen by a
// pass as the GEMM  out(r, n) = sum_k S[r][k] in(k, n),  k the lattice index
// being transformed and n = (other lattice index, column b):
//   "grouped":  addr(k, n) = (n / B) * dim * B + k * B + n % B
//   "row-major": addr(k, n) = k * (other * B) + n
// Pass 1 (x): W grouped -> t1 row-major [ix][iy][b]
// Pass 2 (y): t1 grouped -> t2 row-major [ky][kx][b], scaled by 1 / lambda
// Pass 3 (y): t2 row-major -> t1 grouped [kx][iy][b]
// Pass 4 (x): t1 row-major -> W grouped [iy][ix][b]
// so that every pass reads or writes one side with unit stride along n.
//
// One CTA computes a 128 (n) x up to 256 (r) block of out^T in TMEM:
//   A = in^T tile (128 n x 64 k per K slab), staged by the threads from the
//       vector precision into BF16 shared memory (K-major, no swizzle);
//   B = S tile (r x 64 k), pre-arranged in global memory in exactly the
//       shared-memory layout and fetched by one 1-D bulk copy per slab;
//   D = 128 TMEM lanes (n) x r columns (FP32).
// Two smem stages: the threads stage slab s+1 while the MMAs of slab s run.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cstdint>
#include <mutex>
#include "common.h"
#include "tc.cuh"

namespace qd {

struct GemmTile {
  int dot, m0, n0, pad;
};

constexpr int kTcN = 128;        // data columns (n) per CTA = TMEM lanes
constexpr int kTcK = 64;         // K per shared-memory slab
constexpr int kTcRows = 256;     // transform rows (r) per CTA = TMEM columns (2 CTAs per SM)
constexpr int kTcThreads = 256;
constexpr uint64_t kTcWaitNs = 1000000000ull;   // 1 s bound on every wait
constexpr int kTcABytes = kTcN * kTcK * 2;      // 16 KiB per A stage

__host__ __device__ inline int tc_rpad(int dim) { return (dim + 15) / 16 * 16; }
__host__ __device__ inline int tc_ks(int dim) { return (dim + kTcK - 1) / kTcK; }
__host__ __device__ inline int64_t tc_mat_elems(int dim) {
  return int64_t(tc_rpad(dim)) * tc_ks(dim) * kTcK;
}
__host__ __device__ inline uint32_t tc_tmem_cols(int rows) {
  uint32_t c = 32;
  while (c < uint32_t(rows)) c <<= 1;
  return c;
}

// Dynamic shared-memory layout for a launch whose CTAs hold at most
// `rows_max` transform rows.
struct TcSmem {
  uint32_t a_off[2], b_off[2], lam_off, bar_off, total;
  __host__ __device__ explicit TcSmem(int rows_max) {
    const uint32_t bb = uint32_t(rows_max) * 128u;   // B stage: rows x 64 k x 2 bytes
    a_off[0] = 0;
    a_off[1] = kTcABytes;
    b_off[0] = 2 * kTcABytes;
    b_off[1] = b_off[0] + bb;
    lam_off = b_off[1] + bb;
    bar_off = lam_off + kTcRows * 4;
    total = bar_off + 64;
  }
};

// Bytes of dynamic shared memory to request: the layout, raised so that no
// more CTAs fit on an SM than its 512 TMEM columns can serve at once (an SM
// has 228 KiB of shared memory and reserves 1 KiB per CTA).
inline size_t tc_smem_request(int rows_max) {
  const size_t need = TcSmem(rows_max).total;
  const int allowed = 512 / int(tc_tmem_cols(rows_max));
  const size_t floor_bytes = 233472 / size_t(allowed + 1) + 1 + 128 - 1024;
  return need > floor_bytes ? need : floor_bytes;
}

template <typename T>
__device__ __forceinline__ T from_f32(float v) {
  return T(v);
}
template <>
__device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}

// Two adjacent elements (8-byte / 4-byte / 16-byte aligned pair) as floats.
__device__ __forceinline__ float2 ld_pair(const __nv_bfloat16 *p) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
}
__device__ __forceinline__ float2 ld_pair(const float *p) {
  return *reinterpret_cast<const float2 *>(p);
}
__device__ __forceinline__ float2 ld_pair(const double *p) {
  const double2 d = *reinterpret_cast<const double2 *>(p);
  return make_float2(float(d.x), float(d.y));
}

// out(r, n) = sum_k S[r][k] in(k, n)  [/ (lambda_r(r) + lambda_n(n / B) + shift)]
template <typename TI, typename TO, bool YPASS, bool IN_G, bool OUT_G, bool SCALE>
__global__ void __launch_bounds__(kTcThreads)
dst_tc_kernel(const GemmTile *__restrict__ tiles, const int *__restrict__ active,
              int active_stride, const qd_dst_prec *__restrict__ desc,
              const int32_t *__restrict__ row_off, const uint16_t *__restrict__ mats, int B,
              int rows_max, const TI *__restrict__ in, TO *__restrict__ out, int *err) {
  const GemmTile t = tiles[blockIdx.x];
  // the dot's flag, descriptor and row offset in one round of loads
  const int run = active ? active[size_t(t.dot) * active_stride] : 1;
  const qd_dst_prec d = desc[t.dot];
  const int32_t roff = row_off[t.dot];
  if (!run) return;
  const int dim = YPASS ? d.ny : d.nx;
  const int other = YPASS ? d.nx : d.ny;
  const int ncols = other * B;
  const int KS = tc_ks(dim);
  const int rows = min(kTcRows, tc_rpad(dim) - t.m0);   // multiple of 16
  const uint32_t tcols = tc_tmem_cols(rows);
  const uint16_t *S = mats + (YPASS ? d.sy_off : d.sx_off) + int64_t(t.m0) * KS * kTcK;
  const size_t base = size_t(roff) * B;

  extern __shared__ __align__(1024) uint8_t sm[];
  const TcSmem lay(rows_max);
  uint64_t *bar_full = reinterpret_cast<uint64_t *>(sm + lay.bar_off);
  uint64_t *bar_mma = bar_full + 2;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar_mma + 2);
  float *lam = reinterpret_cast<float *>(sm + lay.lam_off);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    tc::mbar_init(&bar_full[0], 1);
    tc::mbar_init(&bar_full[1], 1);
    tc::mbar_init(&bar_mma[0], 1);
    tc::mbar_init(&bar_mma[1], 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, tcols);
    tc::tmem_relinquish();
  }
  if (SCALE) {
    const float c_r = YPASS ? d.cy : d.cx;
    for (int i = tid; i < rows; i += kTcThreads) {
      const int r = t.m0 + i;
      float v = 0.f;
      if (r < dim) {
        const double sn = sinpi(double(r + 1) / double(2 * (dim + 1)));
        v = float(double(c_r) * 4.0 * sn * sn);
      }
      lam[i] = v;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  // ---- main loop over K slabs ---------------------------------------------
  const size_t in_kstride = IN_G ? size_t(B) : size_t(ncols);
  const uint32_t sA0 = tc::smem_u32(sm + lay.a_off[0]);
  const uint32_t sB0 = tc::smem_u32(sm + lay.b_off[0]);
  const uint32_t lboB = uint32_t(rows) * 16u;     // (rows / 8) core matrices x 128 bytes
  const uint32_t bbytes = uint32_t(rows) * 128u;  // one B slab
  const uint32_t bstage = lay.b_off[1] - lay.b_off[0];
  int issued = 0;    // slabs whose MMAs thread 0 has issued
  int bissued = 0;   // slabs whose operand-B copy thread 0 has issued
  bool fail = false;
  // Operand B of slab s + 1 is fetched as soon as the MMAs of slab s - 1 (the
  // last reader of its stage) are done, right after slab s's MMAs are issued,
  // so that the copy lands while the threads stage operand A of slab s + 1.
  auto issue_b = [&](int s) {   // thread 0
    const int st = s & 1;
    tc::mbar_arrive_expect_tx(&bar_full[st], bbytes);
    tc::bulk_g2s(sm + lay.b_off[0] + st * bstage, S + size_t(s) * rows * kTcK, bbytes,
                 &bar_full[st]);
    bissued = s + 1;
  };
  if (tid == 0) issue_b(0);
  // A slab: the thread's adjacent columns pn, pn + 1 and K chunks pg, pg + 4
  // (8 consecutive k each), both columns of a k loaded with one access (B is
  // even and n0 a multiple of 128, so an even n and n + 1 are adjacent in both
  // layouts and never straddle a group of B).  For row-major input a warp's
  // load then covers a full 128-byte line.  Slab s+1 is loaded into registers
  // while slab s is multiplied.
  const int pn = (tid & 63) * 2, pg = tid >> 6;
  const int np = t.n0 + pn;
  const bool pvalid = np < ncols;   // ncols = other * B is even
  const TI *pin = in + (IN_G ? base + size_t(np / B) * dim * B + (np % B) : base + np);
  float v[4][8];   // v[2 jj + q]: chunk pg + 4 jj, column pn + q
  auto load_a = [&](int s) {
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      const int kc = s * kTcK + (pg + 4 * jj) * 8;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int k = kc + e;
        float2 f = make_float2(0.f, 0.f);
        if (pvalid && k < dim) f = ld_pair(pin + size_t(k) * in_kstride);
        v[2 * jj][e] = f.x;
        v[2 * jj + 1][e] = f.y;
      }
    }
  };
  load_a(0);
  for (int s = 0; s < KS; ++s) {
    const int st = s & 1;
    if (s >= 2 && !tc::mbar_wait(&bar_mma[st], ((s - 2) >> 1) & 1, kTcWaitNs)) fail = true;
    const uint32_t sA = sA0 + uint32_t(st) * kTcABytes, sB = sB0 + uint32_t(st) * bstage;
    uint8_t *a_st = sm + lay.a_off[0] + st * kTcABytes;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = pg + 4 * (j >> 1), nl = pn + (j & 1);   // as loaded above
      uint4 pk;
      uint32_t *w = reinterpret_cast<uint32_t *>(&pk);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v[j][2 * e], v[j][2 * e + 1]);
        w[e] = *reinterpret_cast<const uint32_t *>(&h);
      }
      *reinterpret_cast<uint4 *>(a_st + c * (kTcABytes / 8) + (nl >> 3) * 128 + (nl & 7) * 16) =
          pk;
    }
    if (s + 1 < KS) load_a(s + 1);
    tc::fence_proxy_async_smem();
    fail = __syncthreads_or(fail) != 0;
    if (fail) break;
    if (tid == 0) {
      issued = s + 1;
      if (!tc::mbar_wait(&bar_full[st], (s >> 1) & 1, kTcWaitNs)) {
        fail = true;
      } else {
        tc::fence_after_sync();
#pragma unroll
        for (int kk = 0; kk < kTcK / 16; ++kk) {
          const uint64_t ad = tc::smem_desc(sA + kk * 2 * (kTcABytes / 8), kTcABytes / 8, 128);
          for (int p0 = 0; p0 < rows; p0 += 256) {
            const int np = min(256, rows - p0);
            const uint64_t bd = tc::smem_desc(sB + kk * 2 * lboB + (p0 >> 3) * 128, lboB, 128);
            tc::mma_bf16(tmem + uint32_t(p0), ad, bd, tc::idesc_bf16_f32(128, np),
                         (s > 0 || kk > 0) ? 1u : 0u);
          }
        }
        tc::mma_commit(&bar_mma[st]);
        if (s + 1 < KS) {
          // stage (s + 1) & 1 was last read by the MMAs of slab s - 1
          if (s >= 1 && !tc::mbar_wait(&bar_mma[(s + 1) & 1], ((s - 1) >> 1) & 1, kTcWaitNs))
            fail = true;
          else
            issue_b(s + 1);
        }
      }
    }
  }
  if (!fail) {
    const int last = (KS - 1) & 1;
    if (!tc::mbar_wait(&bar_mma[last], ((KS - 1) >> 1) & 1, kTcWaitNs)) fail = true;
  }
  fail = __syncthreads_or(fail) != 0;
  if (!fail) {
    tc::fence_after_sync();
    // ---- epilogue: TMEM lane quarter (warp & 3), column half (warp >> 2) ---
    const int q = warp & 3, h = warp >> 2;
    const int ne = t.n0 + q * 32 + lane;
    const bool ev = ne < ncols;
    const size_t obase = OUT_G ? base + size_t(ne / B) * dim * B + (ne % B) : base + ne;
    const size_t ostride = OUT_G ? size_t(B) : size_t(ncols);
    float lam_n = 0.f;
    if (SCALE && ev) {
      const double sn = sinpi(double(ne / B + 1) / double(2 * (other + 1)));
      lam_n = float(double(YPASS ? d.cx : d.cy) * 4.0 * sn * sn + double(d.shift));
    }
    for (int c = h; c < rows / 16; c += 2) {
      float a[16];
      tc::tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c * 16), a);
      if (ev) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int r = t.m0 + c * 16 + j;
          if (r < dim) {
            float x = a[j];
            if (SCALE) x = x / (lam[c * 16 + j] + lam_n);
            out[obase + size_t(r) * ostride] = from_f32<TO>(x);
          }
        }
      }
    }
  } else {
    if (tid == 0) {
      atomicOr(err, 1);
      // let this CTA's own bulk copies and MMAs finish before its shared
      // memory and TMEM are released: the last phase armed on each barrier
      // (copies of slabs bissued-1 and bissued-2, MMAs of slabs issued-1 and
      // issued-2; a commit covers all earlier MMAs)
      for (int u = bissued - 2; u < bissued; ++u)
        if (u >= 0) tc::mbar_wait(&bar_full[u & 1], (u >> 1) & 1, kTcWaitNs);
      for (int u = issued - 2; u < issued; ++u)
        if (u >= 0) tc::mbar_wait(&bar_mma[u & 1], (u >> 1) & 1, kTcWaitNs);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, tcols);
}

// Tile tables of the x passes (dim nx, columns ny*B) and y passes (dim ny,
// columns nx*B) for every dot with a preconditioner; rows_x / rows_y receive
// the largest TMEM row block of each.
inline void dst_tiles(int n_dots, const qd_dst_prec *h, int B, GemmTile *tx, int64_t *ntx,
                      GemmTile *ty, int64_t *nty, int *rows_x = nullptr, int *rows_y = nullptr) {
  int64_t a = 0, b = 0;
  int rx = 16, ry = 16;
  for (int d = 0; d < n_dots; ++d) {
    const int nx = h[d].nx, ny = h[d].ny;
    if (nx <= 0 || ny <= 0) continue;
    // row blocks innermost: the CTAs of one data tile run side by side and
    // the later ones read the tile from L2
    for (int n0 = 0; n0 < ny * B; n0 += kTcN)
      for (int m0 = 0; m0 < tc_rpad(nx); m0 += kTcRows) {
        rx = std::max(rx, std::min(kTcRows, tc_rpad(nx) - m0));
        if (tx) tx[a] = GemmTile{d, m0, n0, 0};
        ++a;
      }
    for (int n0 = 0; n0 < nx * B; n0 += kTcN)
      for (int m0 = 0; m0 < tc_rpad(ny); m0 += kTcRows) {
        ry = std::max(ry, std::min(kTcRows, tc_rpad(ny) - m0));
        if (ty) ty[b] = GemmTile{d, m0, n0, 0};
        ++b;
      }
  }
  *ntx = a;
  *nty = b;
  if (rows_x) *rows_x = rx;
  if (rows_y) *rows_y = ry;
}

template <typename TI, typename TO, bool YPASS, bool IN_G, bool OUT_G, bool SCALE>
inline cudaError_t dst_tc_launch(const GemmTile *tiles, int64_t ntiles, int rows_max,
                                 const int *active, int active_stride, const qd_dst_prec *desc,
                                 const int32_t *row_off, const uint16_t *mats, int B,
                                 const TI *in, TO *out, int *err, cudaStream_t s) {
  auto kern = dst_tc_kernel<TI, TO, YPASS, IN_G, OUT_G, SCALE>;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [&] {
    attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448);
  });
  if (attr != cudaSuccess) return attr;
  kern<<<unsigned(ntiles), kTcThreads, tc_smem_request(rows_max), s>>>(
      tiles, active, active_stride, desc, row_off, mats, B, rows_max, in, out, err);
  return cudaGetLastError();
}

// W <- T W (in == out allowed) using tmp1/tmp2 (>= n x B bf16 each).
template <typename TV>
inline cudaError_t dst_apply(const GemmTile *tx, int64_t ntx, int rows_x, const GemmTile *ty,
                             int64_t nty, int rows_y, const int *active, int active_stride,
                             const qd_dst_prec *desc, const int32_t *row_off,
                             const uint16_t *mats, int B, const TV *in, TV *out, void *tmp1,
                             void *tmp2, int *err, cudaStream_t s) {
  if (ntx == 0 || nty == 0) return cudaSuccess;
  using bf = __nv_bfloat16;
  bf *t1 = static_cast<bf *>(tmp1), *t2 = static_cast<bf *>(tmp2);
  cudaError_t e;
  e = dst_tc_launch<TV, bf, false, true, false, false>(tx, ntx, rows_x, active, active_stride,
                                                       desc, row_off, mats, B, in, t1, err, s);
  if (e != cudaSuccess) return e;
  e = dst_tc_launch<bf, bf, true, true, false, true>(ty, nty, rows_y, active, active_stride,
                                                     desc, row_off, mats, B, t1, t2, err, s);
  if (e != cudaSuccess) return e;
  e = dst_tc_launch<bf, bf, true, false, true, false>(ty, nty, rows_y, active, active_stride,
                                                      desc, row_off, mats, B, t2, t1, err, s);
  if (e != cudaSuccess) return e;
  e = dst_tc_launch<bf, TV, false, false, true, false>(tx, ntx, rows_x, active, active_stride,
                                                       desc, row_off, mats, B, t1, out, err, s);
  g_launches.fetch_add(4, std::memory_order_relaxed);
  return e;
}

}  // namespace qd
