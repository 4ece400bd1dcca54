// Open-system eigensolve on the GPU: block LOBPCG on the complex-symmetric
// pencil A = H + i Himag, M (a complex absorbing potential) with every step
// on the device.  The reference solves this pencil densely on the host
// (backend/src/schrodinger.cpp:699-818: a regularised Cholesky of M and
// Eigen's ComplexEigenSolver on the whole matrix); here only the 3b x 3b
// projected problem is dense, and it is solved by hand-written kernels too.
//
// One iteration (columns of the basis S = [X P W] are row-major complex
// blocks [n][3b], with AS = A S and MS = M S beside them):
//   residual      R = AX - MX theta, column norms          cap_resid_kernel
//   precondition  W = T R[:, active] (tensor-core DST of the real kinetic
//                 operator on real and imaginary parts)    qd_dst_precond_apply
//   products      AW, MW                                    qd_cap_spmm
//   Gram          GM = S^H MS, GA = S^H AS (FP64 sums)      cap_gram_kernel
//   orthonormalise  B with B^H GM B = I: Cholesky of the diagonally scaled
//                 Gram matrix in one CTA while its pivots exceed 1e-6, else
//                 SVQB (its Hermitian eigenproblem by the Jacobi kernel)
//   projected problem  C = B^H GA B, Schur form C = Z T Z^H by a Jacobi-like
//                 method for non-Hermitian matrices (G. W. Stewart, SIAM J.
//                 Sci. Stat. Comput. 6 (1985) 853-864): cyclic 2 x 2 unitary
//                 similarity rotations, each zeroing the element below the
//                 diagonal of its 2 x 2 block, in the parallel round-robin
//                 order.  The matrix and Z live in the distributed shared
//                 memory of an 8-CTA cluster (rows split between the CTAs).
//   Ritz pairs    the b eigenvalues of smallest real part, eigenvectors by
//                 back-substitution in T, Y = B Z y, x^H M x = 1
//   update        X = S Y, P = S[:, b:] Y[b:], AP, MP       cap_combine_kernel
//   new products  AX, MX of the new X                        qd_cap_spmm
// The host reads only the b residual norms per iteration (to pick the active
// columns and stop).
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>
#include "common.h"

namespace cg = cooperative_groups;

namespace {

constexpr int kMaxB = 48;            // largest block (3b <= 144)
constexpr int kMaxU = 3 * kMaxB;     // leading dimension of every small matrix
constexpr int kJC = 8;               // CTAs per cluster of the Schur kernel
constexpr int kJRows = kMaxU / kJC;  // rows of Z per CTA (18)
constexpr int kJThreads = 512;
constexpr double kSchurTol = 1e-14;   // |c_qp| <= kSchurTol ||C||_F counts as zero
constexpr int kSchurSweeps = 60;

template <typename T> struct CT;
template <> struct CT<float> { using type = float2; };
template <> struct CT<double> { using type = double2; };

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {   // conj(a) b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  // scaled so that neither |b|^2 nor the products overflow
  const double s = fmax(fabs(b.x), fabs(b.y));
  if (s == 0.0) return make_double2(0.0, 0.0);
  const double bx = b.x / s, by = b.y / s, d = bx * bx + by * by;
  return make_double2((a.x * bx + a.y * by) / (d * s), (a.y * bx - a.x * by) / (d * s));
}
__device__ __forceinline__ double2 csqrt(double2 z) {   // principal branch
  const double r = hypot(z.x, z.y);
  if (r == 0.0) return make_double2(0.0, 0.0);
  const double t = sqrt(0.5 * (r + fabs(z.x)));
  if (z.x >= 0.0) return make_double2(t, z.y / (2.0 * t));
  return make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
template <typename T2> __device__ __forceinline__ T2 from_d2(double2 v);
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) { return make_float2(float(v.x), float(v.y)); }
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }

// 16-byte asynchronous copy of which the first src_bytes come from gmem and
// the rest is zero-filled (gmem 16-byte aligned)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {   // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// ---------------------------------------------------------------------------
// Block initialisation and copies
// ---------------------------------------------------------------------------
template <typename T2>
__global__ void cap_init_kernel(int32_t n, int b, int ld, uint64_t seed, T2 *X) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= int64_t(n) * b) return;
  const int64_t r = i / b;
  const int c = int(i % b);
  const double s = 1.0 / 9007199254740992.0;   // 2^-53
  const double u1 = double(mix64(seed ^ uint64_t(2 * i)) >> 11) * s * 2.0 - 1.0;
  const double u2 = double(mix64(seed ^ uint64_t(2 * i + 1)) >> 11) * s * 2.0 - 1.0;
  X[r * ld + c] = from_d2<T2>(make_double2(u1, u2));
}

template <typename TI2, typename TO2>
__global__ void cap_copy_kernel(int32_t n, int b, const TI2 *in, int ldi, TO2 *out, int ldo) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= int64_t(n) * b) return;
  const int64_t r = i / b;
  const int c = int(i % b);
  out[r * ldo + c] = from_d2<TO2>(to_d2(in[r * ldi + c]));
}

// ---------------------------------------------------------------------------
// Residual R = AX - MX theta (b columns) and per-CTA column norms
// ||R_j||^2, ||MX_j||^2 (FP64); cap_resnorm_kernel sums them in CTA order.
// ---------------------------------------------------------------------------
constexpr int kResBlocks = 592;   // 4 x 148 SMs

template <typename T2>
__global__ void __launch_bounds__(256)
cap_resid_kernel(int32_t n, int b, int ld, const T2 *__restrict__ AX, const T2 *__restrict__ MX,
                 const double2 *__restrict__ theta, T2 *__restrict__ R, double *__restrict__ part) {
  __shared__ double s_r[4][64], s_m[4][64];
  const int c = threadIdx.x & 63, rg = threadIdx.x >> 6;
  double rn = 0.0, mn = 0.0;
  if (c < b) {
    const double2 th = theta[c];
    for (int64_t r = int64_t(blockIdx.x) * 4 + rg; r < n; r += int64_t(gridDim.x) * 4) {
      const double2 a = to_d2(AX[r * ld + c]), m = to_d2(MX[r * ld + c]);
      const double2 q = csub(a, cmul(m, th));
      R[r * b + c] = from_d2<T2>(q);
      rn += cabs2(q);
      mn += cabs2(m);
    }
  }
  s_r[rg][c] = rn;
  s_m[rg][c] = mn;
  __syncthreads();
  if (rg == 0 && c < b) {
    part[size_t(blockIdx.x) * 2 * kMaxB + c] = (s_r[0][c] + s_r[1][c]) + (s_r[2][c] + s_r[3][c]);
    part[size_t(blockIdx.x) * 2 * kMaxB + kMaxB + c] =
        (s_m[0][c] + s_m[1][c]) + (s_m[2][c] + s_m[3][c]);
  }
}

// res_j = ||R_j|| / (max(||MX_j||, 1e-300) max(|theta_j|, eig_scale)); one
// warp per sum (lanes over the CTA partials in a fixed order, then a fixed
// shuffle tree)
__global__ void __launch_bounds__(1024)
cap_resnorm_kernel(int nblk, int b, const double *__restrict__ part,
                   const double2 *__restrict__ theta, double eig_scale, double *__restrict__ res) {
  __shared__ double s_sum[2 * kMaxB];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = warp; q < 2 * b; q += 32) {
    const int off = q < b ? q : kMaxB + (q - b);
    double acc = 0.0;
    for (int k = lane; k < nblk; k += 32) acc += part[size_t(k) * 2 * kMaxB + off];
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) s_sum[q] = acc;
  }
  __syncthreads();
  const int c = threadIdx.x;
  if (c >= b) return;
  const double th = sqrt(cabs2(theta[c]));
  res[c] = sqrt(s_sum[c]) / (fmax(sqrt(s_sum[b + c]), 1e-300) * fmax(th, eig_scale));
}

// out[r][i] = R[r][act[i]] (the active residual columns, contiguous)
template <typename T2>
__global__ void cap_gather_kernel(int32_t n, int b, int m, const int *__restrict__ act,
                                  const T2 *__restrict__ R, T2 *__restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= int64_t(n) * m) return;
  const int64_t r = i / m;
  const int c = int(i % m);
  out[i] = R[r * b + act[c]];
}

// ---------------------------------------------------------------------------
// Gram partials: tiles of GM = S^H MS (upper block triangle, the matrix is
// Hermitian) and GA = S^H AS (all tiles) over row splits.  48 x 48 complex
// tile per CTA, 3 x 3 outputs per thread, rows staged through shared memory
// by a 4-stage cp.async pipeline (16 rows per stage).  FP32 inputs are
// multiplied in FP32 and summed in FP32 over one stage, then in FP64.
// ---------------------------------------------------------------------------
constexpr int kGT = 48;
constexpr int kGRows = 16;
constexpr int kGStages = 4;
constexpr int kGPartTiles = 296;   // row splits x tiles per launch: one wave of 2 CTAs per SM

__device__ __forceinline__ void gram_tile_of(int t, int nt, int &part, int &it, int &jt) {
  const int ngm = nt * (nt + 1) / 2;
  if (t < ngm) {
    part = 0;
    int i = 0, rem = t;
    while (rem >= nt - i) {
      rem -= nt - i;
      ++i;
    }
    it = i;
    jt = i + rem;
  } else {
    part = 1;
    it = (t - ngm) / nt;
    jt = (t - ngm) % nt;
  }
}

template <typename T>
__global__ void __launch_bounds__(256, 2)
cap_gram_kernel(int32_t n, int u, int ld, int rows_per_split,
                const typename CT<T>::type *__restrict__ S, const typename CT<T>::type *__restrict__ MS,
                const typename CT<T>::type *__restrict__ AS, double2 *__restrict__ part_out) {
  using T2 = typename CT<T>::type;
  constexpr int CPR = kGT * int(sizeof(T2)) / 16;     // 16-byte chunks per tile row
  constexpr int TILE = kGRows * kGT;                  // elements per staged tile
  extern __shared__ __align__(16) unsigned char gsm[];
  T2 *sS = reinterpret_cast<T2 *>(gsm);
  T2 *sX = sS + kGStages * TILE;
  const int nt = (u + kGT - 1) / kGT;
  int part, it, jt;
  gram_tile_of(blockIdx.y, nt, part, it, jt);
  const T2 *X2 = part == 0 ? MS : AS;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_split;
  const int64_t r1 = min(int64_t(n), r0 + rows_per_split);
  const int nstage = r1 > r0 ? int((r1 - r0 + kGRows - 1) / kGRows) : 0;
  const int tid = threadIdx.x, ti = tid / 16, tj = tid % 16;
  const int ci0 = it * kGT, cj0 = jt * kGT;

  auto issue = [&](int st) {
    if (st < nstage) {
      T2 *ds = sS + (st % kGStages) * TILE, *dx = sX + (st % kGStages) * TILE;
      const int64_t rb = r0 + int64_t(st) * kGRows;
      for (int e = tid; e < 2 * kGRows * CPR; e += 256) {
        const int which = e / (kGRows * CPR), w = e % (kGRows * CPR);
        const int rr = w / CPR, ch = w % CPR;
        const int64_t r = rb + rr;
        const int c = ch * (16 / int(sizeof(T2)));   // first element of the chunk
        const int col = (which ? cj0 : ci0) + c;
        // bytes of the chunk inside the used columns (the rest is zero-filled)
        const int bytes = r < r1 ? max(0, min(16, (u - col) * int(sizeof(T2)))) : 0;
        const T2 *src = (which ? X2 : S) + (bytes ? r * ld + col : 0);
        cp_async16((which ? dx : ds) + rr * kGT + c, src, bytes);
      }
    }
    cp_async_commit();
  };

  double2 acc[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[a][c] = make_double2(0.0, 0.0);

  for (int st = 0; st < kGStages - 1; ++st) issue(st);
  for (int st = 0; st < nstage; ++st) {
    cp_async_wait<kGStages - 2>();
    __syncthreads();
    issue(st + kGStages - 1);
    const T2 *ps = sS + (st % kGStages) * TILE, *px = sX + (st % kGStages) * TILE;
    if constexpr (sizeof(T) == 8) {
#pragma unroll 4
      for (int rr = 0; rr < kGRows; ++rr) {
        double2 sa[3], xb[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) sa[a] = to_d2(ps[rr * kGT + ti * 3 + a]);
#pragma unroll
        for (int c = 0; c < 3; ++c) xb[c] = to_d2(px[rr * kGT + tj * 3 + c]);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            acc[a][c].x = fma(sa[a].x, xb[c].x, fma(sa[a].y, xb[c].y, acc[a][c].x));
            acc[a][c].y = fma(sa[a].x, xb[c].y, fma(-sa[a].y, xb[c].x, acc[a][c].y));
          }
      }
    } else {
      float2 fa[3][3];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) fa[a][c] = make_float2(0.f, 0.f);
#pragma unroll 4
      for (int rr = 0; rr < kGRows; ++rr) {
        float2 sa[3], xb[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const T2 v = ps[rr * kGT + ti * 3 + a];
          sa[a] = make_float2(float(v.x), float(v.y));
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T2 v = px[rr * kGT + tj * 3 + c];
          xb[c] = make_float2(float(v.x), float(v.y));
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            fa[a][c].x = fmaf(sa[a].x, xb[c].x, fmaf(sa[a].y, xb[c].y, fa[a][c].x));
            fa[a][c].y = fmaf(sa[a].x, xb[c].y, fmaf(-sa[a].y, xb[c].x, fa[a][c].y));
          }
      }
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          acc[a][c].x += double(fa[a][c].x);
          acc[a][c].y += double(fa[a][c].y);
        }
    }
  }
  cp_async_wait<0>();
  double2 *out = part_out + (size_t(blockIdx.x) * gridDim.y + blockIdx.y) * (kGT * kGT);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) out[(ti * 3 + a) * kGT + tj * 3 + c] = acc[a][c];
}

// GM (Hermitian, from the upper tiles; diagonal tiles averaged with their
// conjugate transposes) and GA, [kMaxU][kMaxU], summed over splits in order.
__global__ void cap_gram_reduce_kernel(int u, int nsplit, int ntiles,
                                       const double2 *__restrict__ part, double2 *__restrict__ GM,
                                       double2 *__restrict__ GA) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2 * u * u) return;
  const int which = e / (u * u), w = e % (u * u), i = w / u, j = w % u;
  const int nt = (u + kGT - 1) / kGT, ngm = nt * (nt + 1) / 2;
  auto tile_index = [&](int p, int a, int c) {   // tile of part p at block (a, c)
    if (p == 1) return ngm + a * nt + c;
    return a * nt - a * (a - 1) / 2 + (c - a);    // a <= c
  };
  auto sum = [&](int t, int ii, int jj) {
    double2 s = make_double2(0.0, 0.0);
    for (int k = 0; k < nsplit; ++k) s = cadd(s, part[(size_t(k) * ntiles + t) * (kGT * kGT) + ii * kGT + jj]);
    return s;
  };
  const int ti = i / kGT, tj = j / kGT;
  if (which == 1) {
    GA[i * kMaxU + j] = sum(tile_index(1, ti, tj), i % kGT, j % kGT);
    return;
  }
  double2 g;
  if (ti == tj) {
    const int t = tile_index(0, ti, tj);
    const double2 a = sum(t, i % kGT, j % kGT), b = sum(t, j % kGT, i % kGT);
    g = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
  } else if (ti < tj) {
    g = sum(tile_index(0, ti, tj), i % kGT, j % kGT);
  } else {
    g = cconj(sum(tile_index(0, tj, ti), j % kGT, i % kGT));
  }
  GM[i * kMaxU + j] = g;
}

// ---------------------------------------------------------------------------
// Orthonormaliser by Cholesky (one CTA): Gs = D^-1 GM D^-1 (D = sqrt diag),
// Gs = L L^H, B = D^-1 L^-H (upper triangular, so S B keeps the order of
// S's columns).  Refused (ok = 0) when a diagonal entry is not positive or a
// pivot is <= 1e-6 (condition number of Gs above ~1e6); SVQB then runs.
// Packed lower triangle of Gs in shared memory (u <= 144: 167 KB).
// ---------------------------------------------------------------------------
constexpr size_t kCholSmem = size_t(kMaxU) * (kMaxU + 1) / 2 * sizeof(double2) +
                             2 * kMaxU * sizeof(double2) + kMaxU * sizeof(double) + 64;

__global__ void __launch_bounds__(1024)
cap_chol_kernel(int u, const double2 *__restrict__ GM, double2 *__restrict__ B,
                double *__restrict__ dscale, int *__restrict__ nkeep, int *__restrict__ ok) {
  extern __shared__ __align__(16) unsigned char csm[];
  double2 *L = reinterpret_cast<double2 *>(csm);
  double2 *tmp = L + size_t(kMaxU) * (kMaxU + 1) / 2;
  double *d = reinterpret_cast<double *>(tmp + 2 * kMaxU);
  int *flag = reinterpret_cast<int *>(d + kMaxU);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto at = [&](int i, int j) -> double2 & { return L[i * (i + 1) / 2 + j]; };   // j <= i
  if (tid == 0) *flag = 1;
  __syncthreads();
  for (int i = tid; i < u; i += 1024) {
    const double g = GM[i * kMaxU + i].x;
    d[i] = g > 0.0 ? sqrt(g) : 0.0;
    dscale[i] = d[i];
    if (!(g > 0.0)) *flag = 0;
  }
  __syncthreads();
  if (!*flag) {
    if (tid == 0) *ok = 0;
    return;
  }
  for (int e = tid; e < u * u; e += 1024) {
    const int i = e / u, j = e % u;
    if (j <= i) at(i, j) = cscale(GM[i * kMaxU + j], 1.0 / (d[i] * d[j]));
  }
  __syncthreads();
  for (int j = 0; j < u; ++j) {
    const double piv = at(j, j).x;
    if (!(piv > 1e-6)) {   // uniform: every thread reads the same value
      if (tid == 0) *ok = 0;
      return;
    }
    const double ljj = sqrt(piv);
    __syncthreads();
    if (tid == 0) at(j, j) = make_double2(ljj, 0.0);
    for (int i = j + 1 + tid; i < u; i += 1024) at(i, j) = cscale(at(i, j), 1.0 / ljj);
    __syncthreads();
    for (int i = j + 1 + warp; i < u; i += 32) {
      const double2 lij = at(i, j);
      for (int k = j + 1 + lane; k <= i; k += 32) at(i, k) = csub(at(i, k), cmul(lij, cconj(at(k, j))));
    }
    __syncthreads();
  }
  // in-place inverse of L, last column first:
  // Linv[j+1:, j] = -Linv[j+1:, j+1:] L[j+1:, j] / L[j][j]
  for (int j = u - 1; j >= 0; --j) {
    const double inv = 1.0 / at(j, j).x;
    for (int i = j + 1 + warp; i < u; i += 32) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = j + 1 + lane; k <= i; k += 32) s = cadd(s, cmul(at(i, k), at(k, j)));
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (lane == 0) tmp[i] = s;
    }
    __syncthreads();
    for (int i = j + 1 + tid; i < u; i += 1024) at(i, j) = cscale(tmp[i], -inv);
    if (tid == 0) at(j, j) = make_double2(inv, 0.0);
    __syncthreads();
  }
  // B[i][j] = conj(Linv[j][i]) / d_i for i <= j
  for (int e = tid; e < u * u; e += 1024) {
    const int i = e / u, j = e % u;
    B[i * kMaxU + j] = i <= j ? cscale(cconj(at(j, i)), 1.0 / d[i]) : make_double2(0.0, 0.0);
  }
  if (tid == 0) {
    *nkeep = u;
    *ok = 1;
  }
}

// SVQB input: Gs = Dinv GM Dinv (Dinv = 0 where the diagonal is not positive)
__global__ void cap_svqb_prep_kernel(int u, const int *__restrict__ ok, const double2 *__restrict__ GM,
                                     double *__restrict__ dscale, double2 *__restrict__ J) {
  if (*ok) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= u * u) return;
  const int i = e / u, j = e % u;
  auto dinv = [&](int k) {
    const double g = GM[k * kMaxU + k].x;
    return g > 0.0 ? 1.0 / sqrt(g) : 0.0;
  };
  J[i * kMaxU + j] = cscale(GM[i * kMaxU + j], dinv(i) * dinv(j));
  if (j == 0) dscale[i] = dinv(i);
}

// B = Dinv Z[:, keep] Lambda^-1/2 with keep = lambda > drop * max(lambda)
__global__ void cap_svqb_finish_kernel(int u, double drop, const int *__restrict__ ok,
                                       const double2 *__restrict__ T, const double2 *__restrict__ Z,
                                       const double *__restrict__ dinv, double2 *__restrict__ B,
                                       int *__restrict__ nkeep) {
  if (*ok) return;
  __shared__ int s_col[kMaxU];
  __shared__ double s_lmax;
  const int tid = threadIdx.x;
  if (tid == 0) {
    double lmax = 0.0;
    for (int i = 0; i < u; ++i) lmax = fmax(lmax, T[i * kMaxU + i].x);
    s_lmax = fmax(lmax, 1e-300);
    int m = 0;
    for (int i = 0; i < u; ++i) s_col[i] = T[i * kMaxU + i].x > drop * s_lmax ? m++ : -1;
    *nkeep = m;
  }
  __syncthreads();
  for (int e = tid; e < u * u; e += blockDim.x) {
    const int i = e / u, c = e % u;   // row i of B, source column c of Z
    if (s_col[c] < 0) continue;
    const double lam = T[c * kMaxU + c].x;
    B[i * kMaxU + s_col[c]] = cscale(Z[i * kMaxU + c], dinv[i] / sqrt(lam));
  }
}

// ---------------------------------------------------------------------------
// Small dense complex products on [kMaxU][kMaxU]-strided matrices:
// C (m x nn) = op(A) (m x k) B (k x nn), op(A) = A or A^H.  Dimensions are
// read from device memory where the pointer is given (the kept rank of the
// orthonormaliser is only known on the device).  16 x 16 output tile per CTA.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
cap_small_gemm_kernel(int m, int nn, int k, const int *m_dev, const int *n_dev, const int *k_dev,
                      int adjA, const double2 *__restrict__ A, int lda, const double2 *__restrict__ Bm,
                      int ldb, double2 *__restrict__ Cm, int ldc) {
  if (m_dev) m = *m_dev;
  if (n_dev) nn = *n_dev;
  if (k_dev) k = *k_dev;
  __shared__ double2 sa[16][17], sb[16][17];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int row = blockIdx.y * 16 + ty, col = blockIdx.x * 16 + tx;
  if (blockIdx.y * 16 >= m || blockIdx.x * 16 >= nn) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < k; k0 += 16) {
    {
      const int ar = blockIdx.y * 16 + ty, ak = k0 + tx;   // element (ar, ak) of op(A)
      double2 v = make_double2(0.0, 0.0);
      if (ar < m && ak < k) v = adjA ? cconj(A[ak * lda + ar]) : A[ar * lda + ak];
      sa[ty][tx] = v;
      const int bk = k0 + ty, bc = blockIdx.x * 16 + tx;
      sb[ty][tx] = (bk < k && bc < nn) ? Bm[bk * ldb + bc] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) acc = cadd(acc, cmul(sa[ty][kk], sb[kk][tx]));
    __syncthreads();
  }
  if (row < m && col < nn) Cm[row * ldc + col] = acc;
}

// ---------------------------------------------------------------------------
// Schur form C = Z T Z^H of an n x n complex matrix (n <= 144) by the
// Jacobi-like method for non-Hermitian matrices (Stewart 1985): in each
// round of the parallel round-robin order, every pair (p, q), p < q, gets
// the unitary U whose first column is the eigenvector of the 2 x 2 block
// [[c_pp, c_pq], [c_qp, c_qq]] for the eigenvalue nearer c_pp, and
// C <- U^H C U, Z <- Z U, which zeroes c_qp.  A sweep is N-1 rounds (N = n
// rounded up to even with a decoupled zero row and column); the iteration
// stops after a sweep in which no |c_qp| exceeded rel_tol ||C||_F.  For a
// Hermitian input the result is its eigendecomposition (T diagonal).
//
// Cluster of kJC CTAs.  The pairs are split into kJC contiguous ranges, and
// CTA r keeps the rows of C of the indices paired in its range, so that a
// pair's 2 x 2 block and both of its rows are local.  Round-robin order as
// a ring: index N-1 stays in pair 0, the other indices move one place per
// round (the first member of pair k+1 to pair k, the second member of pair
// k-1 to pair k; pair 0's moving member to pair 1, the last pair's second
// member becomes its first), so only the two rows at each range boundary
// change CTA per round.  Z's rows are split statically (only its columns
// rotate).  Per round:
//   (1) warp 0 forms the rotations of the CTA's pairs and writes them to
//       every CTA; the other warps rotate Z's columns by the previous round's
//       rotations;
//   (2) cluster barrier; each CTA applies U_a^H B U_b to every 2 x 2 block B
//       of its rows (rows of pair a, columns of pair b);
//   (3) the boundary rows go to the neighbours' landing rows; cluster
//       barrier; each CTA moves the landed rows into the freed slots.
// Every thread of every CTA passes the same barriers (the loop bounds and
// the stop test are cluster-uniform).
// ---------------------------------------------------------------------------
struct Rot {
  double2 u1, u2;   // U = [[u1, -conj(u2)], [u2, conj(u1)]]
  int on, p, q, pad;
};

constexpr int kJPairs = kMaxU / 2 / kJC;     // pairs per CTA (9)
constexpr int kJSlots = 2 * kJPairs + 2;     // rows of C per CTA: pairs' rows + 2 landing rows
constexpr int kLandL = 2 * kJPairs, kLandR = 2 * kJPairs + 1;
constexpr size_t kJSmem = size_t(kJSlots) * kMaxU * sizeof(double2) +     // C rows
                          size_t(kJRows) * kMaxU * sizeof(double2) +      // Z rows
                          2 * (kMaxU / 2) * sizeof(Rot) +
                          (2 * kJPairs + kJSlots + 4) * sizeof(int) + 2 * sizeof(double) + 64;

__device__ __forceinline__ Rot make_rot(double2 a, double2 bb, double2 c, double2 d, double thresh2,
                                        int p, int q) {
  Rot R;
  R.u1 = make_double2(1.0, 0.0);
  R.u2 = make_double2(0.0, 0.0);
  R.on = 0;
  R.p = p;
  R.q = q;
  R.pad = 0;
  if (cabs2(c) > thresh2) {
    // eigenvalue lambda of the 2 x 2 block nearer a: with h = (a - d)/2,
    // disc = sqrt(h^2 + b c), lambda - a = b c / g, g the larger of h +- disc
    // (entries are O(||C||), far from the FP64 range limits: plain formulas)
    const double2 h = cscale(csub(a, d), 0.5);
    const double2 z = cadd(cmul(h, h), cmul(bb, c));
    const double r = sqrt(cabs2(z));
    double2 disc = make_double2(0.0, 0.0);
    if (r > 0.0) {
      const double t = sqrt(0.5 * (r + fabs(z.x)));
      const double v = 0.5 * z.y / t;
      disc = z.x >= 0.0 ? make_double2(t, v) : make_double2(fabs(v), copysign(t, z.y));
    }
    const double2 g1 = cadd(h, disc), g2 = csub(h, disc);
    const double2 g = cabs2(g1) >= cabs2(g2) ? g1 : g2;
    const double gg = cabs2(g);
    const double2 delta = gg > 0.0 ? cscale(cmul(cmul(bb, c), cconj(g)), 1.0 / gg) : make_double2(0.0, 0.0);
    // eigenvector [lambda - d, c] = [2h + delta, c] (c != 0)
    const double2 v1 = cadd(cscale(h, 2.0), delta), v2 = c;
    const double inv = rsqrt(cabs2(v1) + cabs2(v2));
    R.u1 = cscale(v1, inv);
    R.u2 = cscale(v2, inv);
    R.on = 1;
  }
  return R;
}

__global__ void __cluster_dims__(kJC, 1, 1) __launch_bounds__(kJThreads, 1)
cap_schur_kernel(int n_fix, const int *__restrict__ n_dev, const int *__restrict__ skip_if_set,
                 const double2 *__restrict__ Cin, int ldi, double2 *__restrict__ Tout,
                 double2 *__restrict__ Zout, int ldo, int max_sweeps, double rel_tol,
                 int *__restrict__ sweeps_out) {
  cg::cluster_group cluster = cg::this_cluster();
  // uniform early exit (every CTA reads the same flag before any barrier)
  if (skip_if_set && *skip_if_set) return;
  const int n = n_dev ? *n_dev : n_fix;
  const int N = n + (n & 1);
  const int M = N - 1;                       // the fixed index
  const int npairs = N / 2, K = npairs - 1;  // K: last pair
  const int P = (npairs + kJC - 1) / kJC;    // pairs per CTA
  const int RZ = (N + kJC - 1) / kJC;        // Z rows per CTA
  const int rank = int(cluster.block_rank());
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  extern __shared__ __align__(16) unsigned char jsm[];
  double2 *Cs = reinterpret_cast<double2 *>(jsm);
  double2 *Zl = Cs + size_t(kJSlots) * kMaxU;
  Rot *rot = reinterpret_cast<Rot *>(Zl + size_t(kJRows) * kMaxU);   // [2][kMaxU / 2]
  int *pos = reinterpret_cast<int *>(rot + 2 * (kMaxU / 2));         // [2 kJPairs] slot of (pair, member)
  int *idx = pos + 2 * kJPairs;                                       // [kJSlots] index held by a slot
  int *s_cnt = idx + kJSlots;                                         // [2] rotations this sweep
  double *s_norm = reinterpret_cast<double *>(s_cnt + 4);
  __shared__ double s_w[kJThreads / 32];
  __shared__ int s_new[2 * kJPairs], s_fill[2][2];

  const int k0 = rank * P, k1 = min(npairs, k0 + P), np = max(0, k1 - k0);
  const int z0 = rank * RZ, nz = max(0, min(RZ, N - z0));
  // round-0 positions: pair 0 = (M, 0), pair k = (k, M - k)
  if (tid < 2 * np) {
    const int k = k0 + tid / 2, m = tid & 1;
    pos[tid] = tid;
    idx[tid] = k == 0 ? (m == 0 ? M : 0) : (m == 0 ? k : M - k);
  }
  if (tid == 0) {
    s_cnt[0] = s_cnt[1] = 0;
    idx[kLandL] = idx[kLandR] = -1;
  }
  __syncthreads();
  double nrm = 0.0;
  for (int e = tid; e < 2 * np * N; e += kJThreads) {
    const int sl = e / N, j = e % N, i = idx[sl];
    const double2 v = (i < n && j < n) ? Cin[size_t(i) * ldi + j] : make_double2(0.0, 0.0);
    Cs[sl * kMaxU + j] = v;
    nrm += cabs2(v);
  }
  for (int e = tid; e < nz * N; e += kJThreads) {
    const int li = e / N, j = e % N;
    Zl[li * kMaxU + j] = make_double2(z0 + li == j ? 1.0 : 0.0, 0.0);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
  if (lane == 0) s_w[warp] = nrm;
  __syncthreads();
  if (tid == 0) {
    double sacc = 0.0;
    for (int w = 0; w < kJThreads / 32; ++w) sacc += s_w[w];
    s_norm[0] = sacc;
  }
  cluster.sync();
  double fro2 = 0.0;
  for (int r = 0; r < kJC; ++r) fro2 += *cluster.map_shared_rank(s_norm, r);
  const double thresh2 = rel_tol * rel_tol * fro2;

  // Z <- Z U for the rotations of one round (rotation table `par`)
  // items (row, pair) spread evenly over threads t0..t0+nt-1; the quotient
  // by npairs in single precision is exact for these small integers
  const float inv_np = 1.0f / float(npairs);
  auto rotate_z = [&](int par, int t0, int nt) {
    for (int e = tid - t0; e < nz * npairs; e += nt) {
      const int li = int((float(e) + 0.5f) * inv_np), k = e - li * npairs;
      const Rot &R = rot[par * (kMaxU / 2) + k];
      if (!R.on) continue;
      double2 *z = Zl + li * kMaxU;
      const double2 x = z[R.p], y = z[R.q];
      z[R.p] = cadd(cmul(x, R.u1), cmul(y, R.u2));
      z[R.q] = csub(cmul(y, cconj(R.u1)), cmul(x, cconj(R.u2)));
    }
  };

  int sweeps = 0, converged = N < 2;
  int g = 0;   // rounds run
  for (int sw = 0; sw < max_sweeps && N >= 2; ++sw) {
    const int cpar = sw & 1;
    for (int rr = 0; rr < N - 1; ++rr, ++g) {
      const int par = g & 1;
      // (1) rotations of my pairs (warp 0), Z by the previous round (others)
      if (warp == 0) {
        if (lane < np) {
          const int k = k0 + lane;
          int sp = pos[2 * lane], sq = pos[2 * lane + 1];
          int p = idx[sp], q = idx[sq];
          if (p > q) {
            const int t = p; p = q; q = t;
            const int u = sp; sp = sq; sq = u;
          }
          const Rot R = make_rot(Cs[sp * kMaxU + p], Cs[sp * kMaxU + q], Cs[sq * kMaxU + p],
                                 Cs[sq * kMaxU + q], thresh2, p, q);
          if (R.on) atomicAdd(&s_cnt[cpar], 1);
          for (int dst = 0; dst < kJC; ++dst) {
            Rot *rp = dst == rank ? rot : cluster.map_shared_rank(rot, dst);
            rp[par * (kMaxU / 2) + k] = R;
          }
        }
      } else if (g > 0) {
        if (tid >= 64) rotate_z(par ^ 1, 64, kJThreads - 64);
      }
      cluster.sync();
      // (2) 2 x 2 blocks of my rows: U_a^H B U_b
      for (int e = tid; e < np * npairs; e += kJThreads) {
        const int t = int((float(e) + 0.5f) * inv_np), kb = e - t * npairs;
        const Rot &Ra = rot[par * (kMaxU / 2) + k0 + t];
        const Rot &Rb = rot[par * (kMaxU / 2) + kb];
        if (!Ra.on && !Rb.on) continue;
        int sp = pos[2 * t], sq = pos[2 * t + 1];
        if (idx[sp] != Ra.p) {
          const int u = sp; sp = sq; sq = u;
        }
        double2 *rp = Cs + sp * kMaxU, *rq = Cs + sq * kMaxU;
        double2 x0 = rp[Rb.p], x1 = rp[Rb.q], y0 = rq[Rb.p], y1 = rq[Rb.q];
        if (Ra.on) {   // rows: [p; q] <- U_a^H [p; q]
          const double2 nx0 = cadd(cmulc(Ra.u1, x0), cmulc(Ra.u2, y0));
          const double2 nx1 = cadd(cmulc(Ra.u1, x1), cmulc(Ra.u2, y1));
          const double2 ny0 = csub(cmul(Ra.u1, y0), cmul(Ra.u2, x0));
          const double2 ny1 = csub(cmul(Ra.u1, y1), cmul(Ra.u2, x1));
          x0 = nx0; x1 = nx1; y0 = ny0; y1 = ny1;
        }
        if (Rb.on) {   // columns: [p' q'] <- [p' q'] U_b
          const double2 cu1 = cconj(Rb.u1), cu2 = cconj(Rb.u2);
          const double2 nx0 = cadd(cmul(x0, Rb.u1), cmul(x1, Rb.u2));
          const double2 nx1 = csub(cmul(x1, cu1), cmul(x0, cu2));
          const double2 ny0 = cadd(cmul(y0, Rb.u1), cmul(y1, Rb.u2));
          const double2 ny1 = csub(cmul(y1, cu1), cmul(y0, cu2));
          x0 = nx0; x1 = nx1; y0 = ny0; y1 = ny1;
        }
        if (kb == k0 + t && Ra.on) y0 = make_double2(0.0, 0.0);   // the zeroed c_qp
        rp[Rb.p] = x0;
        rp[Rb.q] = x1;
        rq[Rb.p] = y0;
        rq[Rb.q] = y1;
      }
      __syncthreads();
      // (3) ring shift: member 0 of my first pair goes left, member 1 of my
      // last pair goes right (each to the neighbour's landing row)
      const bool out_l = np > 0 && k0 >= 1, out_r = np > 0 && k1 - 1 < K;
      if (out_l || out_r) {
        for (int e = tid; e < 2 * N; e += kJThreads) {
          const int side = e / N, j = e % N;
          if (side == 0 ? !out_l : !out_r) continue;
          const int src = side == 0 ? pos[0] : pos[2 * (np - 1) + 1];
          const int dst_rank = side == 0 ? rank - 1 : rank + 1;
          double2 *peer = cluster.map_shared_rank(Cs, dst_rank);
          peer[(side == 0 ? kLandR : kLandL) * kMaxU + j] = Cs[src * kMaxU + j];
          if (j == 0) cluster.map_shared_rank(idx, dst_rank)[side == 0 ? kLandR : kLandL] = idx[src];
        }
      }
      if (K >= 1) {
        // new slot of every position (k, m), k in my range (one thread each):
        // the source position's slot if local, else a landing row, moved into
        // the slot freed by the row that left on the same side
        if (tid < 2) s_fill[tid][0] = -1;
        __syncthreads();
        if (tid < 2 * np) {
          const int t = tid >> 1, m = tid & 1, k = k0 + t;
          int sk, sm;   // source position
          if (m == 0) {
            if (k == 0) { sk = 0; sm = 0; }
            else if (k < K) { sk = k + 1; sm = 0; }
            else { sk = K; sm = 1; }
          } else {
            if (k == 0) { sk = 1; sm = 0; }
            else if (k == 1) { sk = 0; sm = 1; }
            else { sk = k - 1; sm = 1; }
          }
          int slot;
          if (sk >= k0 && sk < k1) {
            slot = pos[2 * (sk - k0) + sm];
          } else if (sk < k0) {   // arrives from the left
            slot = pos[0];
            s_fill[0][0] = kLandL;
            s_fill[0][1] = slot;
          } else {                 // arrives from the right
            slot = pos[2 * (np - 1) + 1];
            s_fill[1][0] = kLandR;
            s_fill[1][1] = slot;
          }
          s_new[tid] = slot;
        }
      }
      cluster.sync();
      // landed rows into the freed slots, then the new positions
      if (K >= 1) {
        for (int e = tid; e < 2 * N; e += kJThreads) {
          const int side = e / N, j = e % N;
          const int from = s_fill[side][0];
          if (from < 0) continue;
          const int to = s_fill[side][1];
          Cs[to * kMaxU + j] = Cs[from * kMaxU + j];
          if (j == 0) idx[to] = idx[from];
        }
        if (tid < 2 * np) pos[tid] = s_new[tid];
      }
      __syncthreads();
    }
    ++sweeps;
    int total = 0;
    for (int r = 0; r < kJC; ++r) total += cluster.map_shared_rank(s_cnt, r)[cpar];
    cluster.sync();   // every CTA has read the counters
    if (tid == 0) s_cnt[cpar] = 0;
    __syncthreads();
    if (total == 0) {
      converged = 1;
      break;
    }
  }
  if (g > 0) rotate_z((g - 1) & 1, 0, kJThreads);   // the last round's rotations
  __syncthreads();
  for (int e = tid; e < 2 * np * N; e += kJThreads) {
    const int sl = e / N, j = e % N;
    const int s_ = pos[sl], i = idx[s_];
    if (i < n && j < n) Tout[size_t(i) * ldo + j] = Cs[s_ * kMaxU + j];
  }
  for (int e = tid; e < nz * N; e += kJThreads) {
    const int li = e / N, j = e % N, i = z0 + li;
    if (i < n && j < n) Zout[size_t(i) * ldo + j] = Zl[li * kMaxU + j];
  }
  if (rank == 0 && tid == 0 && sweeps_out) {
    sweeps_out[0] = sweeps;
    sweeps_out[1] = converged;
  }
  cluster.sync();   // no CTA leaves while a peer may still write to it
}

// ---------------------------------------------------------------------------
// Ritz pairs from the Schur form: the b diagonal entries of T of smallest
// real part (ties by position), in that order.
// ---------------------------------------------------------------------------
__global__ void cap_select_kernel(const int *__restrict__ n_dev, int b, const double2 *__restrict__ T,
                                  int *__restrict__ sel, double2 *__restrict__ theta,
                                  int *__restrict__ status) {
  const int n = *n_dev;
  const int i = threadIdx.x;
  if (i == 0 && n < b) atomicOr(status, 2);
  if (i >= n) return;
  const double key = T[i * kMaxU + i].x;
  if (key != key) atomicOr(status, 4);
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const double kj = T[j * kMaxU + j].x;
    rank += (kj < key) || (kj == key && j < i);
  }
  if (rank < b) {
    sel[rank] = i;
    theta[rank] = T[i * kMaxU + i];
  }
}

// Eigenvector of T for the selected diagonal position (back-substitution,
// one CTA per Ritz pair, T's leading upper triangle staged column-major in
// shared memory), then V[:, j] = Z y.
__global__ void __launch_bounds__(256)
cap_schur_vec_kernel(const int *__restrict__ n_dev, int b, const int *__restrict__ sel,
                     const double2 *__restrict__ T, const double2 *__restrict__ Z,
                     double2 *__restrict__ V) {
  extern __shared__ __align__(16) unsigned char vsm[];
  double2 *Tc = reinterpret_cast<double2 *>(vsm);                 // packed columns 0..pos
  double2 *y = Tc + size_t(kMaxU) * (kMaxU + 1) / 2;               // [kMaxU]
  const int n = *n_dev;
  const int j = blockIdx.x;
  if (j >= b || n < b) return;
  const int pos = sel[j];
  const int tid = threadIdx.x;
  for (int e = tid; e < (pos + 1) * (pos + 1); e += 256) {
    const int r = e / (pos + 1), c = e % (pos + 1);
    if (r <= c) Tc[c * (c + 1) / 2 + r] = T[r * kMaxU + c];
  }
  __syncthreads();
  const double2 lam = Tc[pos * (pos + 1) / 2 + pos];
  double tmax = 0.0;
  for (int i = 0; i <= pos; ++i) tmax = fmax(tmax, sqrt(cabs2(Tc[i * (i + 1) / 2 + i])));
  const double smin = fmax(2.220446049250313e-16 * tmax, 1e-300);
  // y[pos] = 1; rhs = -T[0:pos, pos]; solve upwards
  for (int i = tid; i < pos; i += 256) y[i] = cscale(Tc[pos * (pos + 1) / 2 + i], -1.0);
  if (tid == 0) y[pos] = make_double2(1.0, 0.0);
  __syncthreads();
  for (int i = pos - 1; i >= 0; --i) {
    double2 den = csub(Tc[i * (i + 1) / 2 + i], lam);
    if (sqrt(cabs2(den)) < smin) den = make_double2(smin, 0.0);
    const double2 yi = cdiv(y[i], den);   // every thread computes the same value
    __syncthreads();
    if (tid == 0) y[i] = yi;
    for (int l = tid; l < i; l += 256) y[l] = csub(y[l], cmul(Tc[i * (i + 1) / 2 + l], yi));
    __syncthreads();
  }
  for (int l = tid; l < n; l += 256) {
    double2 s = make_double2(0.0, 0.0);
    for (int i = 0; i <= pos; ++i) s = cadd(s, cmul(Z[l * kMaxU + i], y[i]));
    V[l * kMaxB + j] = s;
  }
}

// Y[:, j] /= sqrt(Re y_j^H GM y_j) (Hermitian M-normalised Ritz vectors);
// Yf receives the FP32 copy.
__global__ void __launch_bounds__(256)
cap_ritz_norm_kernel(int u, int b, const double2 *__restrict__ GM, double2 *__restrict__ Y,
                     float2 *__restrict__ Yf) {
  __shared__ double s_part[256];
  __shared__ double s_scale;
  const int j = blockIdx.x, tid = threadIdx.x;
  double acc = 0.0;
  for (int a = tid; a < u; a += 256) {
    double2 g = make_double2(0.0, 0.0);
    for (int c = 0; c < u; ++c) g = cadd(g, cmul(GM[a * kMaxU + c], Y[c * kMaxB + j]));
    acc += cmulc(Y[a * kMaxB + j], g).x;
  }
  s_part[tid] = acc;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int t = 0; t < 256; ++t) s += s_part[t];
    s_scale = 1.0 / sqrt(fmax(s, 1e-300));
  }
  __syncthreads();
  for (int a = tid; a < u; a += 256) {
    const double2 v = cscale(Y[a * kMaxB + j], s_scale);
    Y[a * kMaxB + j] = v;
    Yf[a * kMaxB + j] = make_float2(float(v.x), float(v.y));
  }
}

// ---------------------------------------------------------------------------
// Block update out[r][0:b] = in[r][k0:K] Y[k0:K][0:b] for up to four
// (in, out, k0) parts at once (blockIdx.y): X = S Y, P = S[:, b:] Y[b:],
// AP = AS[:, b:] Y[b:], MP = MS[:, b:] Y[b:].  64 rows x 48 columns per CTA,
// 4 x 3 outputs per thread, K in chunks of 16 through shared memory.
// ---------------------------------------------------------------------------
template <typename T2> struct CombineArgs {
  const T2 *in[4];
  T2 *out[4];
  int k0[4];
};

template <typename T>
__global__ void __launch_bounds__(256)
cap_combine_kernel(int32_t n, int K, int b, int ld, CombineArgs<typename CT<T>::type> args,
                   const typename CT<T>::type *__restrict__ Y) {
  using T2 = typename CT<T>::type;
  __shared__ T2 sa[64][17];
  __shared__ T2 sy[16][kMaxB];
  // constant-index selection keeps the parameter block out of local memory
  const int part = blockIdx.y;
  const T2 *in = part == 0 ? args.in[0] : part == 1 ? args.in[1] : part == 2 ? args.in[2] : args.in[3];
  T2 *out = part == 0 ? args.out[0] : part == 1 ? args.out[1] : part == 2 ? args.out[2] : args.out[3];
  const int k0 = part == 0 ? args.k0[0] : part == 1 ? args.k0[1] : part == 2 ? args.k0[2] : args.k0[3];
  const int tid = threadIdx.x, tr = tid / 16, tc = tid % 16;
  const int64_t rbase = int64_t(blockIdx.x) * 64;
  double2 acc[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[a][c] = make_double2(0.0, 0.0);
  for (int kc = k0; kc < K; kc += 16) {
    for (int e = tid; e < 64 * 16; e += 256) {
      const int rr = e / 16, kk = e % 16;
      const int64_t r = rbase + rr;
      sa[rr][kk] = (r < n && kc + kk < K) ? in[r * ld + kc + kk] : from_d2<T2>(make_double2(0.0, 0.0));
    }
    for (int e = tid; e < 16 * kMaxB; e += 256) {
      const int kk = e / kMaxB, c = e % kMaxB;
      sy[kk][c] = (kc + kk < K && c < b) ? Y[(kc + kk) * kMaxB + c] : from_d2<T2>(make_double2(0.0, 0.0));
    }
    __syncthreads();
    if constexpr (sizeof(T) == 8) {
#pragma unroll 4
      for (int kk = 0; kk < 16; ++kk) {
        double2 av[4], yv[3];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = to_d2(sa[tr * 4 + a][kk]);
#pragma unroll
        for (int c = 0; c < 3; ++c) yv[c] = to_d2(sy[kk][tc * 3 + c]);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            acc[a][c].x = fma(av[a].x, yv[c].x, fma(-av[a].y, yv[c].y, acc[a][c].x));
            acc[a][c].y = fma(av[a].x, yv[c].y, fma(av[a].y, yv[c].x, acc[a][c].y));
          }
      }
    } else {
      float2 fa[4][3];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) fa[a][c] = make_float2(0.f, 0.f);
#pragma unroll 4
      for (int kk = 0; kk < 16; ++kk) {
        float2 av[4], yv[3];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const T2 v = sa[tr * 4 + a][kk];
          av[a] = make_float2(float(v.x), float(v.y));
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T2 v = sy[kk][tc * 3 + c];
          yv[c] = make_float2(float(v.x), float(v.y));
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            fa[a][c].x = fmaf(av[a].x, yv[c].x, fmaf(-av[a].y, yv[c].y, fa[a][c].x));
            fa[a][c].y = fmaf(av[a].x, yv[c].y, fmaf(av[a].y, yv[c].x, fa[a][c].y));
          }
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          acc[a][c].x += double(fa[a][c].x);
          acc[a][c].y += double(fa[a][c].y);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int64_t r = rbase + tr * 4 + a;
    if (r >= n) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int col = tc * 3 + c;
      if (col < b) out[r * ld + col] = from_d2<T2>(acc[a][c]);
    }
  }
}

// ---------------------------------------------------------------------------
// Final quantities of the converged block: bilinear x^T A x, x^T M x, then
// ||A x - E M x||^2 and ||M x||^2 (per-CTA partials summed in CTA order).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
cap_bilinear_kernel(int32_t n, int b, int ld, const double2 *__restrict__ X,
                    const double2 *__restrict__ AX, const double2 *__restrict__ MX,
                    const double2 *__restrict__ E, double2 *__restrict__ part) {
  // E == nullptr: part = (x^T A x, x^T M x); else (||Ax - E Mx||^2, ||Mx||^2)
  __shared__ double2 s_a[4][64], s_m[4][64];
  const int c = threadIdx.x & 63, rg = threadIdx.x >> 6;
  double2 sa = make_double2(0.0, 0.0), sm = make_double2(0.0, 0.0);
  if (c < b) {
    const double2 e = E ? E[c] : make_double2(0.0, 0.0);
    for (int64_t r = int64_t(blockIdx.x) * 4 + rg; r < n; r += int64_t(gridDim.x) * 4) {
      const double2 x = X[r * ld + c], a = AX[r * ld + c], m = MX[r * ld + c];
      if (E) {
        sa.x += cabs2(csub(a, cmul(e, m)));
        sm.x += cabs2(m);
      } else {
        sa = cadd(sa, cmul(x, a));
        sm = cadd(sm, cmul(x, m));
      }
    }
  }
  s_a[rg][c] = sa;
  s_m[rg][c] = sm;
  __syncthreads();
  if (rg == 0 && c < b) {
    part[size_t(blockIdx.x) * 2 * kMaxB + c] = cadd(cadd(s_a[0][c], s_a[1][c]), cadd(s_a[2][c], s_a[3][c]));
    part[size_t(blockIdx.x) * 2 * kMaxB + kMaxB + c] =
        cadd(cadd(s_m[0][c], s_m[1][c]), cadd(s_m[2][c], s_m[3][c]));
  }
}

__global__ void cap_sum_kernel(int nblk, int b, const double2 *__restrict__ part, double2 *__restrict__ out) {
  const int c = threadIdx.x;
  if (c >= 2 * kMaxB) return;
  double2 s = make_double2(0.0, 0.0);
  for (int k = 0; k < nblk; ++k) s = cadd(s, part[size_t(k) * 2 * kMaxB + c]);
  out[c] = s;
}

// Xout[:, t] = X[:, pick[t]] * scale[t]
__global__ void cap_output_kernel(int32_t n, int k, int ld, const double2 *__restrict__ X,
                                  const int *__restrict__ pick, const double2 *__restrict__ scale,
                                  double2 *__restrict__ Xout) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= int64_t(n) * k) return;
  const int64_t r = i / k;
  const int t = int(i % k);
  Xout[i] = cmul(X[r * ld + pick[t]], scale[t]);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <auto Kern>
cudaError_t smem_opt_in(size_t bytes) {
  static std::once_flag once;
  static cudaError_t e = cudaSuccess;
  std::call_once(once, [&] { e = cudaFuncSetAttribute(Kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)); });
  return e;
}

struct Blocks {            // one precision's double-buffered S, AS, MS
  void *S[2], *AS[2], *MS[2];
};

struct Work {
  Blocks b64, b32;
  void *R, *pin, *pout, *dst;
  size_t dst_bytes;
  double2 *gpart;
  double2 *GM, *GA, *Bm, *J, *T, *Z, *tmp, *C, *Y, *V;
  float2 *Yf;
  double *dscale, *rpart, *res;
  double2 *theta, *bpart, *bsum, *E, *scale;
  int *nkeep, *ok, *status, *sel, *act, *pick, *sweeps;
};

size_t carve(qd::Arena &ar, int32_t n, int b, bool mixed, size_t dst_bytes, Work &w) {
  const size_t blk = size_t(n) * 3 * b;
  for (int i = 0; i < 2; ++i) {
    w.b64.S[i] = ar.take<double2>(blk);
    w.b64.AS[i] = ar.take<double2>(blk);
    w.b64.MS[i] = ar.take<double2>(blk);
    w.b32.S[i] = mixed ? ar.take<float2>(blk) : nullptr;
    w.b32.AS[i] = mixed ? ar.take<float2>(blk) : nullptr;
    w.b32.MS[i] = mixed ? ar.take<float2>(blk) : nullptr;
  }
  w.R = ar.take<double2>(size_t(n) * b);
  w.pin = ar.take<double2>(size_t(n) * b);
  w.pout = ar.take<double2>(size_t(n) * b);
  w.dst_bytes = dst_bytes;
  w.dst = dst_bytes ? ar.take<unsigned char>(dst_bytes) : nullptr;
  w.gpart = ar.take<double2>(size_t(kGPartTiles) * kGT * kGT);
  const size_t sq = size_t(kMaxU) * kMaxU;
  w.GM = ar.take<double2>(sq);
  w.GA = ar.take<double2>(sq);
  w.Bm = ar.take<double2>(sq);
  w.J = ar.take<double2>(sq);
  w.T = ar.take<double2>(sq);
  w.Z = ar.take<double2>(sq);
  w.tmp = ar.take<double2>(sq);
  w.C = ar.take<double2>(sq);
  w.Y = ar.take<double2>(size_t(kMaxU) * kMaxB);
  w.V = ar.take<double2>(size_t(kMaxU) * kMaxB);
  w.Yf = ar.take<float2>(size_t(kMaxU) * kMaxB);
  w.dscale = ar.take<double>(kMaxU);
  w.rpart = ar.take<double>(size_t(kResBlocks) * 2 * kMaxB);
  w.res = ar.take<double>(kMaxB);
  w.theta = ar.take<double2>(kMaxB);
  w.bpart = ar.take<double2>(size_t(kResBlocks) * 2 * kMaxB);
  w.bsum = ar.take<double2>(2 * kMaxB);
  w.E = ar.take<double2>(kMaxB);
  w.scale = ar.take<double2>(kMaxB);
  w.nkeep = ar.take<int>(1);
  w.ok = ar.take<int>(1);
  w.status = ar.take<int>(1);
  w.sel = ar.take<int>(kMaxB);
  w.act = ar.take<int>(kMaxB);
  w.pick = ar.take<int>(kMaxB);
  w.sweeps = ar.take<int>(2);   // largest sweep count, all converged
  return ar.used;
}

struct Problem {
  int32_t n;
  const int32_t *rowptr, *col;
  const void *H, *G, *M;        // FP64
  const void *H32, *G32, *M32;  // FP32 copies (mixed form)
  const qd_dst_prec *prec;      // host descriptor (nullptr: no preconditioner)
  const void *prec_mats;
  int b, nev;
  double eig_scale;
  cudaStream_t s;
};

unsigned grid_for(int64_t count, int threads) { return unsigned((count + threads - 1) / threads); }

// One precision's LOBPCG run.  On entry X (columns 0..b-1 of cur.S) holds the
// start; on exit cur holds the final block, theta and res the last Ritz
// values and residuals.
template <typename T>
int lobpcg_run(const Problem &P, Work &w, Blocks &bl, int &cur, double tol, int max_iter,
               int stall, double drop, std::vector<double> &res, int &iters, int *sweeps_max,
               int *schur_unconverged) {
  using T2 = typename CT<T>::type;
  const int n = P.n, b = P.b, ld = 3 * b;
  const bool f32 = sizeof(T) == 4;
  cudaStream_t s = P.s;
  const void *H = f32 ? P.H32 : P.H, *G = f32 ? P.G32 : P.G, *M = f32 ? P.M32 : P.M;
  auto S = [&](int i) { return static_cast<T2 *>(bl.S[i]); };
  auto AS = [&](int i) { return static_cast<T2 *>(bl.AS[i]); };
  auto MS = [&](int i) { return static_cast<T2 *>(bl.MS[i]); };
  auto spmm = [&](int blk, int c0, int m) {
    return qd_cap_spmm(n, m, f32 ? 1 : 0, P.rowptr, P.col, H, G, M, S(blk) + c0, ld, AS(blk) + c0,
                       MS(blk) + c0, ld, s);
  };
  QD_CUDA_TRY(smem_opt_in<cap_gram_kernel<T>>(size_t(2) * kGStages * kGRows * kGT * sizeof(T2)));
  QD_CUDA_TRY(smem_opt_in<cap_chol_kernel>(kCholSmem));
  QD_CUDA_TRY(smem_opt_in<cap_schur_kernel>(kJSmem));
  QD_CUDA_TRY(smem_opt_in<cap_schur_vec_kernel>(size_t(kMaxU) * (kMaxU + 1) / 2 * sizeof(double2) +
                                                kMaxU * sizeof(double2)));

  // Rayleigh-Ritz on span S[:, :u] of block `blk`: Y (FP64 and FP32 copies), theta
  auto rayleigh_ritz = [&](int blk, int u) -> int {
    const int nt = (u + kGT - 1) / kGT, ntiles = nt * (nt + 1) / 2 + nt * nt;
    int nsplit = std::max(1, std::min(kGPartTiles / ntiles, int((int64_t(n) + 1023) / 1024)));
    int rps = int((int64_t(n) + nsplit - 1) / nsplit);
    rps = (rps + kGRows - 1) / kGRows * kGRows;
    nsplit = int((int64_t(n) + rps - 1) / rps);
    cap_gram_kernel<T><<<dim3(nsplit, ntiles), 256, size_t(2) * kGStages * kGRows * kGT * sizeof(T2), s>>>(
        n, u, ld, rps, S(blk), MS(blk), AS(blk), w.gpart);
    QD_CHECK_LAUNCH();
    cap_gram_reduce_kernel<<<grid_for(2 * u * u, 256), 256, 0, s>>>(u, nsplit, ntiles, w.gpart, w.GM, w.GA);
    QD_CHECK_LAUNCH();
    cap_chol_kernel<<<1, 1024, kCholSmem, s>>>(u, w.GM, w.Bm, w.dscale, w.nkeep, w.ok);
    QD_CHECK_LAUNCH();
    cap_svqb_prep_kernel<<<grid_for(u * u, 256), 256, 0, s>>>(u, w.ok, w.GM, w.dscale, w.J);
    QD_CHECK_LAUNCH();
    cap_schur_kernel<<<kJC, kJThreads, kJSmem, s>>>(u, nullptr, w.ok, w.J, kMaxU, w.T, w.Z, kMaxU,
                                                    kSchurSweeps, kSchurTol, nullptr);
    QD_CHECK_LAUNCH();
    cap_svqb_finish_kernel<<<1, 256, 0, s>>>(u, drop, w.ok, w.T, w.Z, w.dscale, w.Bm, w.nkeep);
    QD_CHECK_LAUNCH();
    // C = B^H GA B  (u' = nkeep columns of B)
    const dim3 g1((kMaxU + 15) / 16, (u + 15) / 16), g2((kMaxU + 15) / 16, (kMaxU + 15) / 16);
    cap_small_gemm_kernel<<<g1, 256, 0, s>>>(u, 0, u, nullptr, w.nkeep, nullptr, 0, w.GA, kMaxU, w.Bm,
                                             kMaxU, w.tmp, kMaxU);
    QD_CHECK_LAUNCH();
    cap_small_gemm_kernel<<<g2, 256, 0, s>>>(0, 0, u, w.nkeep, w.nkeep, nullptr, 1, w.Bm, kMaxU, w.tmp,
                                             kMaxU, w.C, kMaxU);
    QD_CHECK_LAUNCH();
    cap_schur_kernel<<<kJC, kJThreads, kJSmem, s>>>(0, w.nkeep, nullptr, w.C, kMaxU, w.T, w.Z, kMaxU,
                                                    kSchurSweeps, kSchurTol, w.sweeps);
    QD_CHECK_LAUNCH();
    cap_select_kernel<<<1, kMaxU, 0, s>>>(w.nkeep, b, w.T, w.sel, w.theta, w.status);
    QD_CHECK_LAUNCH();
    cap_schur_vec_kernel<<<b, 256, size_t(kMaxU) * (kMaxU + 1) / 2 * sizeof(double2) + kMaxU * sizeof(double2), s>>>(
        w.nkeep, b, w.sel, w.T, w.Z, w.V);
    QD_CHECK_LAUNCH();
    // Y = B V (u x b)
    const dim3 g3((b + 15) / 16, (u + 15) / 16);
    cap_small_gemm_kernel<<<g3, 256, 0, s>>>(u, b, 0, nullptr, nullptr, w.nkeep, 0, w.Bm, kMaxU, w.V,
                                             kMaxB, w.Y, kMaxB);
    QD_CHECK_LAUNCH();
    cap_ritz_norm_kernel<<<b, 256, 0, s>>>(u, b, w.GM, w.Y, w.Yf);
    QD_CHECK_LAUNCH();
    return QD_OK;
  };
  // nxt.X = S Y, and with_p: nxt.P = S[:, b:u] Y[b:], nxt.AP, nxt.MP
  auto combine = [&](int c, int nx, int u, bool with_p) -> int {
    CombineArgs<T2> a{};
    a.in[0] = S(c);
    a.out[0] = S(nx);
    a.k0[0] = 0;
    a.in[1] = S(c);
    a.out[1] = S(nx) + b;
    a.k0[1] = b;
    a.in[2] = AS(c);
    a.out[2] = AS(nx) + b;
    a.k0[2] = b;
    a.in[3] = MS(c);
    a.out[3] = MS(nx) + b;
    a.k0[3] = b;
    const T2 *Yt = f32 ? reinterpret_cast<const T2 *>(w.Yf) : reinterpret_cast<const T2 *>(w.Y);
    cap_combine_kernel<T><<<dim3(grid_for(n, 64), with_p ? 4 : 1), 256, 0, s>>>(n, u, b, ld, a, Yt);
    QD_CHECK_LAUNCH();
    return QD_OK;
  };

  int st;
  QD_CUDA_TRY(cudaMemsetAsync(w.status, 0, sizeof(int), s));
  if ((st = spmm(cur, 0, b)) != QD_OK) return st;
  if ((st = rayleigh_ritz(cur, b)) != QD_OK) return st;
  if ((st = combine(cur, cur ^ 1, b, false)) != QD_OK) return st;
  cur ^= 1;
  if ((st = spmm(cur, 0, b)) != QD_OK) return st;
  int npc = 0;
  double best = INFINITY;
  int since = 0;
  res.assign(b, INFINITY);
  std::vector<int> act;
  iters = 0;
  for (int it = 1; it <= max_iter; ++it) {
    iters = it;
    cap_resid_kernel<T2><<<kResBlocks, 256, 0, s>>>(n, b, ld, AS(cur), MS(cur), w.theta,
                                                    static_cast<T2 *>(w.R), w.rpart);
    QD_CHECK_LAUNCH();
    cap_resnorm_kernel<<<1, 1024, 0, s>>>(kResBlocks, b, w.rpart, w.theta, P.eig_scale, w.res);
    QD_CHECK_LAUNCH();
    int hstatus = 0, hsweeps[2] = {0, 1};
    QD_CUDA_TRY(cudaMemcpyAsync(res.data(), w.res, b * sizeof(double), cudaMemcpyDeviceToHost, s));
    QD_CUDA_TRY(cudaMemcpyAsync(&hstatus, w.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    QD_CUDA_TRY(cudaMemcpyAsync(hsweeps, w.sweeps, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    QD_CUDA_TRY(cudaStreamSynchronize(s));
    if (sweeps_max) *sweeps_max = std::max(*sweeps_max, hsweeps[0]);
    if (!hsweeps[1]) ++*schur_unconverged;
    if (hstatus) return QD_ERR_BREAKDOWN;
    double worst = 0.0;
    bool finite = true;
    for (int j = 0; j < P.nev; ++j) {
      worst = std::max(worst, res[j]);
      finite = finite && std::isfinite(res[j]);
    }
    if (!finite) return QD_ERR_BREAKDOWN;
    if (worst <= tol) break;
    if (stall) {
      if (worst < 0.9 * best) {
        best = worst;
        since = 0;
      } else if (++since >= stall) {
        break;
      }
    }
    act.clear();
    for (int j = 0; j < b; ++j)
      if (res[j] > tol) act.push_back(j);
    if (act.size() < 2) act = {b - 2, b - 1};
    const int m = int(act.size());
    const int w0 = b + npc;
    QD_CUDA_TRY(cudaMemcpyAsync(w.act, act.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
    // W = T R[:, act] into S[:, w0:w0+m]
    if (P.prec) {
      cap_gather_kernel<T2><<<grid_for(int64_t(n) * m, 256), 256, 0, s>>>(
          n, b, m, w.act, static_cast<const T2 *>(w.R), static_cast<T2 *>(w.pin));
      QD_CHECK_LAUNCH();
      const int32_t ro[2] = {0, n};
      st = qd_dst_precond_apply(1, ro, 2 * m, f32 ? 1 : 0, P.prec, P.prec_mats, w.pin, w.pout, w.dst,
                                w.dst_bytes, s);
      if (st != QD_OK) return st;
      cap_copy_kernel<T2, T2><<<grid_for(int64_t(n) * m, 256), 256, 0, s>>>(
          n, m, static_cast<const T2 *>(w.pout), m, S(cur) + w0, ld);
      QD_CHECK_LAUNCH();
    } else {
      cap_gather_kernel<T2><<<grid_for(int64_t(n) * m, 256), 256, 0, s>>>(
          n, b, m, w.act, static_cast<const T2 *>(w.R), static_cast<T2 *>(w.pin));
      QD_CHECK_LAUNCH();
      cap_copy_kernel<T2, T2><<<grid_for(int64_t(n) * m, 256), 256, 0, s>>>(
          n, m, static_cast<const T2 *>(w.pin), m, S(cur) + w0, ld);
      QD_CHECK_LAUNCH();
    }
    if ((st = spmm(cur, w0, m)) != QD_OK) return st;
    const int u = b + npc + m;
    if ((st = rayleigh_ritz(cur, u)) != QD_OK) return st;
    if ((st = combine(cur, cur ^ 1, u, true)) != QD_OK) return st;
    cur ^= 1;
    npc = b;
    if ((st = spmm(cur, 0, b)) != QD_OK) return st;
  }
  return QD_OK;
}

}  // namespace

extern "C" int qd_cap_lobpcg_workspace_size(int32_t n, int b, int precision, const qd_dst_prec *h_prec,
                                            size_t *bytes) {
  if (n < 1 || b < 2 || b > kMaxB || b % 2 || !bytes ||
      (precision != QD_PREC_FP64 && precision != QD_PREC_MIXED))
    return QD_ERR_INVALID;
  size_t dst = 0;
  if (h_prec) {
    const int32_t ro[2] = {0, n};
    const int st = qd_dst_precond_workspace_size(1, ro, 2 * b, h_prec, &dst);
    if (st != QD_OK) return st;
  }
  qd::Arena ar(nullptr, 0);
  Work w;
  *bytes = carve(ar, n, b, precision == QD_PREC_MIXED, dst, w);
  return QD_OK;
}

extern "C" int qd_cap_lobpcg_solve(int32_t n, const int32_t *d_rowptr, const int32_t *d_col,
                                   const double *d_H, const double *d_Himag, const double *d_M,
                                   const float *d_H32, const float *d_Himag32, const float *d_M32,
                                   const qd_dst_prec *h_prec, const void *d_prec_mats, int b, int nev,
                                   int k, double sigma, double tol, double tol32, int max_iter,
                                   int precision, double eig_scale, uint64_t seed, const void *d_X0,
                                   double *h_E, void *d_Xout, double *h_res, qd_cap_info *h_info,
                                   void *d_work, size_t work_bytes, void *stream) {
  if (n < 1 || b < 2 || b > kMaxB || b % 2 || nev < 1 || nev > b || k < 1 || k > nev || max_iter < 1 ||
      !d_rowptr || !d_col || !d_H || !d_M || !h_E || !d_Xout || !h_res || !h_info || !d_work ||
      (precision != QD_PREC_FP64 && precision != QD_PREC_MIXED) || !(tol > 0.0))
    return QD_ERR_INVALID;
  const bool mixed = precision == QD_PREC_MIXED;
  if (mixed && (!d_H32 || !d_M32 || (d_Himag && !d_Himag32))) return QD_ERR_INVALID;
  if (h_prec && !d_prec_mats) return QD_ERR_INVALID;
  size_t dst = 0;
  if (h_prec) {
    const int32_t ro[2] = {0, n};
    const int st = qd_dst_precond_workspace_size(1, ro, 2 * b, h_prec, &dst);
    if (st != QD_OK) return st;
  }
  qd::Arena ar(d_work, work_bytes);
  Work w;
  const size_t need = carve(ar, n, b, mixed, dst, w);
  if (need > work_bytes || !w.res) return QD_ERR_WORKSPACE;
  Problem P{n, d_rowptr, d_col, d_H, d_Himag, d_M, d_H32, d_Himag32, d_M32, h_prec, d_prec_mats,
            b, nev, eig_scale, static_cast<cudaStream_t>(stream)};
  cudaStream_t s = P.s;
  const int ld = 3 * b;
  std::memset(h_info, 0, sizeof(*h_info));
  QD_CUDA_TRY(cudaMemsetAsync(w.theta, 0, kMaxB * sizeof(double2), s));
  QD_CUDA_TRY(cudaMemsetAsync(w.sweeps, 0, 2 * sizeof(int), s));
  std::vector<double> res;
  int st, cur64 = 0, sweeps = 0, unconv = 0;
  if (mixed) {
    int cur32 = 0, it32 = 0;
    cap_init_kernel<float2><<<grid_for(int64_t(n) * b, 256), 256, 0, s>>>(
        n, b, ld, seed, static_cast<float2 *>(w.b32.S[0]));
    QD_CHECK_LAUNCH();
    st = lobpcg_run<float>(P, w, w.b32, cur32, tol32, max_iter, 8, 1e-6, res, it32, &sweeps, &unconv);
    if (st != QD_OK) return st;
    double r32 = 0.0;
    for (int j = 0; j < nev; ++j) r32 = std::max(r32, res[j]);
    h_info->fp32_residual = r32;
    h_info->iters_fp32 = it32;
    cap_copy_kernel<float2, double2><<<grid_for(int64_t(n) * b, 256), 256, 0, s>>>(
        n, b, static_cast<const float2 *>(w.b32.S[cur32]), ld, static_cast<double2 *>(w.b64.S[0]), ld);
    QD_CHECK_LAUNCH();
  } else if (d_X0) {
    cap_copy_kernel<double2, double2><<<grid_for(int64_t(n) * b, 256), 256, 0, s>>>(
        n, b, static_cast<const double2 *>(d_X0), b, static_cast<double2 *>(w.b64.S[0]), ld);
    QD_CHECK_LAUNCH();
  } else {
    cap_init_kernel<double2><<<grid_for(int64_t(n) * b, 256), 256, 0, s>>>(
        n, b, ld, seed, static_cast<double2 *>(w.b64.S[0]));
    QD_CHECK_LAUNCH();
  }
  int it64 = 0;
  st = lobpcg_run<double>(P, w, w.b64, cur64, tol, max_iter, 0, 1e-14, res, it64, &sweeps, &unconv);
  if (st != QD_OK) return st;
  h_info->iters_fp64 = it64;
  h_info->schur_sweeps_max = sweeps;
  h_info->schur_unconverged = unconv;

  // bilinear Rayleigh quotients, x^T M x = 1 normalisation, residuals
  const double2 *X = static_cast<const double2 *>(w.b64.S[cur64]);
  const double2 *AX = static_cast<const double2 *>(w.b64.AS[cur64]);
  const double2 *MX = static_cast<const double2 *>(w.b64.MS[cur64]);
  cap_bilinear_kernel<<<kResBlocks, 256, 0, s>>>(n, b, ld, X, AX, MX, nullptr, w.bpart);
  QD_CHECK_LAUNCH();
  cap_sum_kernel<<<1, 2 * kMaxB, 0, s>>>(kResBlocks, b, w.bpart, w.bsum);
  QD_CHECK_LAUNCH();
  std::vector<std::complex<double>> sums(2 * kMaxB), theta(kMaxB);
  QD_CUDA_TRY(cudaMemcpyAsync(sums.data(), w.bsum, 2 * kMaxB * sizeof(double2), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaMemcpyAsync(theta.data(), w.theta, kMaxB * sizeof(double2), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<std::complex<double>> E(b), sc(b);
  for (int j = 0; j < b; ++j) {
    E[j] = sums[j] / sums[kMaxB + j];
    sc[j] = 1.0 / std::sqrt(sums[kMaxB + j]);
  }
  QD_CUDA_TRY(cudaMemcpyAsync(w.E, E.data(), b * sizeof(double2), cudaMemcpyHostToDevice, s));
  cap_bilinear_kernel<<<kResBlocks, 256, 0, s>>>(n, b, ld, X, AX, MX, w.E, w.bpart);
  QD_CHECK_LAUNCH();
  cap_sum_kernel<<<1, 2 * kMaxB, 0, s>>>(kResBlocks, b, w.bpart, w.bsum);
  QD_CHECK_LAUNCH();
  QD_CUDA_TRY(cudaMemcpyAsync(sums.data(), w.bsum, 2 * kMaxB * sizeof(double2), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<double> rres(b);
  for (int j = 0; j < b; ++j)
    rres[j] = std::sqrt(sums[j].real()) / (std::sqrt(sums[kMaxB + j].real()) * std::abs(E[j]));
  // the k converged pairs nearest sigma, and whether they are certified
  std::vector<int> conv;
  for (int j = 0; j < nev; ++j)
    if (res[j] <= tol) conv.push_back(j);
  std::vector<int> order(conv);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    return std::abs(E[a] - sigma) < std::abs(E[c] - sigma);
  });
  if (int(order.size()) > k) order.resize(k);
  double dk = order.empty() ? INFINITY : 0.0, bound = INFINITY, rmax = order.empty() ? INFINITY : 0.0;
  for (int j : order) {
    dk = std::max(dk, std::abs(E[j] - sigma));
    rmax = std::max(rmax, rres[j]);
  }
  for (int j = 0; j < b; ++j)
    if (!(j < nev && res[j] <= tol)) bound = std::min(bound, theta[j].real() - sigma);
  const int npick = int(order.size());
  h_info->converged = int(conv.size());
  h_info->selected = npick;
  h_info->complete = (npick == k && dk < bound) ? 1 : 0;
  h_info->kth_distance = dk;
  h_info->unconverged_bound = bound;
  h_info->max_residual = rmax;
  std::vector<std::complex<double>> scale(npick);
  for (int t = 0; t < npick; ++t) {
    h_E[2 * t] = E[order[t]].real();
    h_E[2 * t + 1] = E[order[t]].imag();
    h_res[t] = rres[order[t]];
    scale[t] = sc[order[t]];
  }
  if (npick) {
    QD_CUDA_TRY(cudaMemcpyAsync(w.pick, order.data(), npick * sizeof(int), cudaMemcpyHostToDevice, s));
    QD_CUDA_TRY(cudaMemcpyAsync(w.scale, scale.data(), npick * sizeof(double2), cudaMemcpyHostToDevice, s));
    cap_output_kernel<<<grid_for(int64_t(n) * npick, 256), 256, 0, s>>>(
        n, npick, ld, X, w.pick, w.scale, static_cast<double2 *>(d_Xout));
    QD_CHECK_LAUNCH();
  }
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  const bool all = it64 < max_iter || [&] {
    for (int j = 0; j < nev; ++j)
      if (!(res[j] <= tol)) return false;
    return true;
  }();
  return all ? QD_OK : QD_ERR_NOT_CONVERGED;
}

// Schur form of one small complex matrix (n <= 144) with the cluster kernel
// above: T upper triangular, Z unitary, C = Z T Z^H.  Row-major, leading
// dimensions ldc (input) and ldt (outputs).
extern "C" int qd_complex_schur(int n, const void *d_C, int ldc, void *d_T, void *d_Z, int ldt,
                                int max_sweeps, int *h_sweeps, void *stream) {
  if (n < 1 || n > kMaxU || ldc < n || ldt < n || !d_C || !d_T || !d_Z || max_sweeps < 1)
    return QD_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  QD_CUDA_TRY(smem_opt_in<cap_schur_kernel>(kJSmem));
  int *d_sw = nullptr;
  QD_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&d_sw), 2 * sizeof(int), s));
  cap_schur_kernel<<<kJC, kJThreads, kJSmem, s>>>(n, nullptr, nullptr, static_cast<const double2 *>(d_C),
                                                  ldc, static_cast<double2 *>(d_T),
                                                  static_cast<double2 *>(d_Z), ldt, max_sweeps,
                                                  kSchurTol, d_sw);
  cudaError_t e = cudaGetLastError();
  QD_LAUNCHED();
  int sw[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(sw, d_sw, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(d_sw, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return QD_ERR_CUDA;
  if (h_sweeps) *h_sweeps = sw[0];
  return sw[1] ? QD_OK : QD_ERR_NOT_CONVERGED;
}
