// Batched LOBPCG for the lowest eigenpairs of H x = E M x on a block-diagonal
// batch of independent finite-element problems (one "dot" per block).
//
// Replaces the reference eigensolves: eigsh(H, k, M, which='SM')
// (qdsim_cython/solvers/schrodinger_solver.pyx:447-453), the dense LLT +
// SelfAdjointEigenSolver of EigenSolver::solve (backend/src/solver.cpp:84-128)
// and the densify + cusolverDnZhegvd path (backend/src/gpu_eigensolver.cu:
// 139-238, a stub in the reference build).
//
// Layout: all dots' rows are concatenated; every vector block is row-major
// (n_total x B).  Rows are cut into chunks of kChunkRows rows that never span
// two dots; every row-parallel kernel runs one CTA per chunk and returns at
// once for a dot that has converged, so one launch serves the whole batch and
// the work of uneven dots is balanced by the hardware scheduler.
//
// Per iteration (S = [X W P], products kept in HS = [HX HW HP], MS = [MX MW MP]):
//   gram   : per chunk, A_c = S^T HS and B_c = S^T MS (3B x 3B), FP64 accumulation
//   rr     : per dot (one CTA), A = sum_c A_c, B = sum_c B_c; Cholesky of the
//            column-scaled B, C = L^-1 A L^-T, cyclic Jacobi eigensolve of C,
//            Ritz coefficients Y -- all FP64 in shared memory
//   update : per chunk, X = S Y, P = [W P] Y_wp, same for HS/MS, residual
//            W = HX - MX Theta and its per-column norms
//   spmm   : HW = H W, MW = M W (FP64 accumulation)
// Every kRefresh iterations HX, MX, HP, MP are recomputed from X and P.
//
// Precision: QD_PREC_FP64 stores vectors in FP64.  QD_PREC_MIXED runs the
// same iteration with FP32 vector storage and FP32 update arithmetic (matrix
// values, SpMM accumulation and Gram sums stay FP64) until the FP32 residual
// criterion or stagnation, then converts X to FP64 and finishes in FP64.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "common.h"
#include "spmm.cuh"

namespace {

constexpr int kChunkRows = 2048;
constexpr int kMaxB = 16;
constexpr int kMaxM = 3 * kMaxB;
constexpr int kRefresh32 = 20;
constexpr int kRefresh64 = 40;
constexpr int kStagWindow = 40;
constexpr double kTol32 = 5e-5;

struct Chunk {
  int dot, begin, end, pad;
};

struct DotState {
  int active;       // iterating in the current phase
  int has_p;        // P block is populated
  int iters;        // total iterations (all phases)
  int iters_phase;  // iterations in the current phase
  int iters32;      // iterations spent in the FP32 phase
  int status;       // 0 running, 1 converged, 2 breakdown, 3 iteration cap
  int stag;         // iterations without 20% improvement (FP32 phase)
  int have_res;     // residual norms of the current X are available
  int chunk0, chunk1;
  double best;      // best max relative residual in this phase
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

__device__ inline uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

template <typename TV, int B>
__global__ void init_kernel(const Chunk *chunks, const int32_t *row_off, uint64_t seed, TV *X,
                            TV *W, TV *P, TV *HW, TV *MW, TV *HP, TV *MP) {
  const Chunk ch = chunks[blockIdx.x];
  const int r0 = row_off[ch.dot];
  for (int idx = threadIdx.x; idx < (ch.end - ch.begin) * B; idx += blockDim.x) {
    const int r = ch.begin + idx / B, j = idx % B;
    const uint64_t h = splitmix64(seed * 0x100000001b3ull + uint64_t(r - r0) * B + j);
    const double u = double(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    const size_t o = size_t(r) * B + j;
    X[o] = TV(u);
    W[o] = P[o] = HW[o] = MW[o] = HP[o] = MP[o] = TV(0);
  }
}

template <typename TV, int B>
__global__ void zero_aux_kernel(const Chunk *chunks, TV *W, TV *P, TV *HW, TV *MW, TV *HP, TV *MP) {
  const Chunk ch = chunks[blockIdx.x];
  for (int idx = threadIdx.x; idx < (ch.end - ch.begin) * B; idx += blockDim.x) {
    const size_t o = size_t(ch.begin) * B + idx;
    W[o] = P[o] = HW[o] = MW[o] = HP[o] = MP[o] = TV(0);
  }
}

template <int B>
__global__ void convert_kernel(const Chunk *chunks, const float *X32, double *X64) {
  const Chunk ch = chunks[blockIdx.x];
  for (int idx = threadIdx.x; idx < (ch.end - ch.begin) * B; idx += blockDim.x) {
    const size_t o = size_t(ch.begin) * B + idx;
    X64[o] = double(X32[o]);
  }
}

template <typename TV, int B>
__global__ void spmm_chunk_kernel(const Chunk *chunks, const DotState *st,
                                  const int32_t *__restrict__ rowptr,
                                  const int32_t *__restrict__ col, const double *__restrict__ H,
                                  const double *__restrict__ M, const TV *__restrict__ X,
                                  TV *__restrict__ HX, TV *__restrict__ MX) {
  constexpr int G = B / 4;
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].active) return;
  const int sub = threadIdx.x / G, g = threadIdx.x % G;
  const int rpp = blockDim.x / G;
  for (int r = ch.begin + sub; r < ch.end; r += rpp)
    qd::spmm_row<TV, B, true>(r, g, rowptr, col, H, M, X, HX, MX);
}

// ---------------------------------------------------------------------------
// Gram partials: per chunk A_c = S^T HS, B_c = S^T MS  (m = 3B, full m x m)
// ---------------------------------------------------------------------------

template <int B> struct GramCfg {
  static constexpr int m = 3 * B;
  static constexpr int NB = m / 4;
  static constexpr int NBLK = NB * NB;
  static constexpr int RG = (256 / NBLK) > 0 ? (256 / NBLK) : 1;
  static constexpr int SUB = 32;
  static constexpr int THREADS = ((NBLK * RG + 31) / 32) * 32;
};

template <typename TV, int B>
__global__ void __launch_bounds__(GramCfg<B>::THREADS)
gram_kernel(const Chunk *chunks, const DotState *st, const TV *X, const TV *W, const TV *P,
            const TV *HX, const TV *HW, const TV *HP, const TV *MX, const TV *MW, const TV *MP,
            double *partial) {
  using C = GramCfg<B>;
  constexpr int m = C::m, NB = C::NB, NBLK = C::NBLK, RG = C::RG, SUB = C::SUB;
  constexpr int STAGE_BYTES = 3 * SUB * m * int(sizeof(TV));
  constexpr int RED_BYTES = (RG > 1) ? NBLK * 32 * 8 : 8;
  constexpr int RAW = STAGE_BYTES > RED_BYTES ? STAGE_BYTES : RED_BYTES;
  __shared__ __align__(16) unsigned char raw[RAW];
  TV *sS = reinterpret_cast<TV *>(raw);
  TV *sH = sS + SUB * m;
  TV *sM = sH + SUB * m;

  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].active) return;
  const int tid = threadIdx.x;
  const bool worker = tid < NBLK * RG;
  const int blk = tid % NBLK, rg = tid / NBLK;
  const int bi = blk / NB, bj = blk % NB;
  double aH[4][4], aM[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) aH[a][b] = aM[a][b] = 0.0;

  const TV *srcS[3] = {X, W, P};
  const TV *srcH[3] = {HX, HW, HP};
  const TV *srcM[3] = {MX, MW, MP};
  for (int r0 = ch.begin; r0 < ch.end; r0 += SUB) {
    const int nr = min(SUB, ch.end - r0);
    for (int idx = tid; idx < SUB * m; idx += blockDim.x) {
      const int row = idx / m, c = idx % m;
      const int blkc = c / B, cc = c % B;
      TV s = TV(0), h = TV(0), mm = TV(0);
      if (row < nr) {
        const size_t o = size_t(r0 + row) * B + cc;
        s = srcS[blkc][o];
        h = srcH[blkc][o];
        mm = srcM[blkc][o];
      }
      sS[idx] = s;
      sH[idx] = h;
      sM[idx] = mm;
    }
    __syncthreads();
    if (worker) {
      // products in the storage precision, summed over this sub-tile, then
      // added into FP64 accumulators (FP32: exact products are not needed in
      // the FP32 phase; the FP64 phase runs this with TV = double).
      TV tH[4][4], tM[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) tH[a][b] = tM[a][b] = TV(0);
      for (int row = rg; row < nr; row += RG) {
        TV sa[4], hb[4], mb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          sa[a] = sS[row * m + 4 * bi + a];
          hb[a] = sH[row * m + 4 * bj + a];
          mb[a] = sM[row * m + 4 * bj + a];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            tH[a][b] = fma(sa[a], hb[b], tH[a][b]);
            tM[a][b] = fma(sa[a], mb[b], tM[a][b]);
          }
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          aH[a][b] += double(tH[a][b]);
          aM[a][b] += double(tM[a][b]);
        }
    }
    __syncthreads();
  }
  double *out = partial + size_t(blockIdx.x) * 2 * m * m;
  if (RG > 1) {
    double *red = reinterpret_cast<double *>(raw);
    for (int g = 1; g < RG; ++g) {
      if (worker && rg == g) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            red[blk * 32 + a * 4 + b] = aH[a][b];
            red[blk * 32 + 16 + a * 4 + b] = aM[a][b];
          }
      }
      __syncthreads();
      if (worker && rg == 0) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            aH[a][b] += red[blk * 32 + a * 4 + b];
            aM[a][b] += red[blk * 32 + 16 + a * 4 + b];
          }
      }
      __syncthreads();
    }
  }
  if (worker && rg == 0) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int i = 4 * bi + a, j = 4 * bj + b;
        out[i * m + j] = aH[a][b];
        out[m * m + i * m + j] = aM[a][b];
      }
  }
}

// ---------------------------------------------------------------------------
// Rayleigh-Ritz per dot (FP64, one CTA of 256 threads, m <= 48)
// ---------------------------------------------------------------------------

struct RRParams {
  int k;
  int phase32;     // 1: FP32 phase (stagnation allowed, scaled residual)
  double tol;      // relative residual tolerance for this phase
  int max_iter;    // total iteration cap per dot
};

template <int B>
__global__ void __launch_bounds__(256)
rr_kernel(DotState *st, const double *partial, const double *norms, double *theta,
          double *coef, double *relres, RRParams prm) {
  constexpr int m = 3 * B;
  extern __shared__ double sm[];
  double *sA = sm;             // m*m
  double *sB = sA + m * m;     // m*m  (B, then its Cholesky factor L)
  double *sT = sB + m * m;     // m*m  (L^-1)
  double *sZ = sT + m * m;     // m*m  (temp, then eigenvectors)
  double *sD = sZ + m * m;     // m    column scaling
  double *sE = sD + m;         // m    eigenvalues
  double *sR = sE + m;         // B    relative residuals
  __shared__ int s_flag, s_fail, s_sel[kMaxM];
  __shared__ double s_red[256];

  const int d = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  DotState &s = st[d];
  if (!s.active) return;
  double *th = theta + size_t(d) * B;
  if (tid == 0) s_flag = 0;
  __syncthreads();

  // 1. convergence test on the residual norms of the current X
  if (s.have_res) {
    if (tid < B) {
      double rr = 0.0, mx = 0.0;
      for (int c = s.chunk0; c < s.chunk1; ++c) {
        rr += norms[size_t(c) * 2 * B + tid];
        mx += norms[size_t(c) * 2 * B + B + tid];
      }
      double scale = fabs(th[tid]);
      if (prm.phase32) scale = fmax(scale, fabs(th[B - 1] - th[0]));
      scale = fmax(scale, 1e-300);
      const double rel = sqrt(rr / fmax(mx, 1e-300)) / scale;
      sR[tid] = rel;
      relres[size_t(d) * B + tid] = rel;
    }
    __syncthreads();
    if (tid == 0) {
      double worst = 0.0;
      for (int j = 0; j < prm.k; ++j) worst = fmax(worst, isfinite(sR[j]) ? sR[j] : 1e300);
      int stop = 0;
      if (worst <= prm.tol) {
        stop = 1;
        if (!prm.phase32) s.status = 1;
      } else if (prm.phase32) {
        if (worst < 0.8 * s.best) {
          s.best = worst;
          s.stag = 0;
        } else if (++s.stag >= kStagWindow) {
          stop = 1;
        }
      }
      if (!stop && s.iters >= prm.max_iter) {
        stop = 1;
        s.status = prm.phase32 ? 0 : 3;
      }
      if (stop) {
        s.active = 0;
        s_flag = 1;
      }
    }
    __syncthreads();
    if (s_flag) return;
  }

  // 2. Gram matrices summed over the dot's chunks (fixed order)
  for (int idx = tid; idx < m * m; idx += nt) {
    double a = 0.0, b = 0.0;
    for (int c = s.chunk0; c < s.chunk1; ++c) {
      a += partial[size_t(c) * 2 * m * m + idx];
      b += partial[size_t(c) * 2 * m * m + m * m + idx];
    }
    sA[idx] = a;
    sZ[idx] = b;   // keep the raw B for a retry without P
  }
  __syncthreads();
  int has_p = s.has_p;
  for (int attempt = 0; attempt < 2; ++attempt) {
    // symmetrise, drop P if requested, scale columns
    for (int idx = tid; idx < m * m; idx += nt) {
      const int i = idx / m, j = idx % m;
      double a = 0.5 * (sA[i * m + j] + sA[j * m + i]);
      double b = 0.5 * (sZ[i * m + j] + sZ[j * m + i]);
      if (!has_p && (i >= 2 * B || j >= 2 * B)) a = b = 0.0;
      sT[idx] = a;        // temporarily the symmetric A
      sB[idx] = b;
    }
    __syncthreads();
    // column scaling from the diagonal of B
    double dmax = 0.0;
    for (int i = 0; i < m; ++i) dmax = fmax(dmax, sB[i * m + i]);
    if (tid < m) {
      const double bii = sB[tid * m + tid];
      sD[tid] = (bii > 1e-26 * dmax && isfinite(bii)) ? rsqrt(bii) : 0.0;
    }
    __syncthreads();
    double amax = 0.0;
    for (int i = 0; i < m; ++i) amax = fmax(amax, fabs(sT[i * m + i]) * sD[i] * sD[i]);
    __syncthreads();   // every thread has read the unscaled diagonal
    for (int idx = tid; idx < m * m; idx += nt) {
      const int i = idx / m, j = idx % m;
      double a = sT[idx] * sD[i] * sD[j];
      double b = sB[idx] * sD[i] * sD[j];
      if (i == j && sD[i] == 0.0) {
        b = 1.0;
        a = 1e6 * (amax + 1.0);   // decoupled (null) column: far above the spectrum
      }
      sT[idx] = a;
      sB[idx] = b;
    }
    if (tid == 0) s_fail = 0;
    __syncthreads();
    // Cholesky of B in place (lower)
    for (int j = 0; j < m; ++j) {
      if (tid == 0) {
        const double piv = sB[j * m + j];
        if (!(piv > 1e-13)) s_fail = 1;
        else sB[j * m + j] = sqrt(piv);
      }
      __syncthreads();
      if (s_fail) break;
      const double ljj = sB[j * m + j];
      for (int i = j + 1 + tid; i < m; i += nt) sB[i * m + j] /= ljj;
      __syncthreads();
      const int rem = m - j - 1;
      for (int idx = tid; idx < rem * rem; idx += nt) {
        const int i = j + 1 + idx / rem, l = j + 1 + idx % rem;
        if (l <= i) sB[i * m + l] -= sB[i * m + j] * sB[l * m + j];
      }
      __syncthreads();
    }
    if (!s_fail) break;
    if (!has_p) break;
    has_p = 0;   // retry without the P block
    __syncthreads();
  }
  if (s_fail) {
    if (tid == 0) {
      s.active = 0;
      s.status = 2;
    }
    return;
  }
  // move A (scaled) to sA; L^-1 into sT
  for (int idx = tid; idx < m * m; idx += nt) sA[idx] = sT[idx];
  __syncthreads();
  if (tid < m) {
    const int j = tid;
    for (int i = 0; i < m; ++i) {
      if (i < j) {
        sT[i * m + j] = 0.0;
        continue;
      }
      double sum = (i == j) ? 1.0 : 0.0;
      for (int l = j; l < i; ++l) sum -= sB[i * m + l] * sT[l * m + j];
      sT[i * m + j] = sum / sB[i * m + i];
    }
  }
  __syncthreads();
  // Z = A L^-T ; C = L^-1 Z  (C into sB, which is free now)
  for (int idx = tid; idx < m * m; idx += nt) {
    const int i = idx / m, j = idx % m;
    double sum = 0.0;
    for (int l = 0; l <= j; ++l) sum += sA[i * m + l] * sT[j * m + l];
    sZ[idx] = sum;
  }
  __syncthreads();
  for (int idx = tid; idx < m * m; idx += nt) {
    const int i = idx / m, j = idx % m;
    double sum = 0.0;
    for (int l = 0; l <= i; ++l) sum += sT[i * m + l] * sZ[l * m + j];
    sB[idx] = sum;
  }
  __syncthreads();
  for (int idx = tid; idx < m * m; idx += nt) {
    const int i = idx / m, j = idx % m;
    sA[idx] = 0.5 * (sB[i * m + j] + sB[j * m + i]);
    sZ[idx] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  // cyclic Jacobi with round-robin pairing (m even)
  __shared__ double s_c[kMaxM / 2], s_s[kMaxM / 2];
  __shared__ int s_p[kMaxM / 2], s_q[kMaxM / 2];
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0, fro = 0.0;
    for (int idx = tid; idx < m * m; idx += nt) {
      const int i = idx / m, j = idx % m;
      const double v = sA[idx] * sA[idx];
      fro += v;
      if (i != j) off += v;
    }
    s_red[tid] = off;
    __syncthreads();
    for (int w = nt / 2; w > 0; w >>= 1) {
      if (tid < w) s_red[tid] += s_red[tid + w];
      __syncthreads();
    }
    off = s_red[0];
    __syncthreads();
    s_red[tid] = fro;
    __syncthreads();
    for (int w = nt / 2; w > 0; w >>= 1) {
      if (tid < w) s_red[tid] += s_red[tid + w];
      __syncthreads();
    }
    fro = s_red[0];
    __syncthreads();
    if (off <= 1e-30 * fro) break;
    for (int round = 0; round < m - 1; ++round) {
      if (tid < m / 2) {
        int p, q;
        if (tid == 0) {
          p = 0;
          q = 1 + (round % (m - 1));
        } else {
          p = 1 + ((tid + round) % (m - 1));
          q = 1 + ((m - 1 - tid + round) % (m - 1));
        }
        if (p > q) {
          const int t = p; p = q; q = t;
        }
        const double apq = sA[p * m + q];
        double c = 1.0, sn = 0.0;
        if (fabs(apq) > 1e-300) {
          const double tau = (sA[q * m + q] - sA[p * m + p]) / (2.0 * apq);
          const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = rsqrt(1.0 + t * t);
          sn = t * c;
        }
        s_c[tid] = c;
        s_s[tid] = sn;
        s_p[tid] = p;
        s_q[tid] = q;
      }
      __syncthreads();
      for (int idx = tid; idx < (m / 2) * m; idx += nt) {   // rows
        const int t = idx / m, j = idx % m;
        const int p = s_p[t], q = s_q[t];
        const double c = s_c[t], sn = s_s[t];
        const double a = sA[p * m + j], b = sA[q * m + j];
        sA[p * m + j] = c * a - sn * b;
        sA[q * m + j] = sn * a + c * b;
      }
      __syncthreads();
      for (int idx = tid; idx < (m / 2) * m; idx += nt) {   // columns (and Z)
        const int t = idx / m, i = idx % m;
        const int p = s_p[t], q = s_q[t];
        const double c = s_c[t], sn = s_s[t];
        const double a = sA[i * m + p], b = sA[i * m + q];
        sA[i * m + p] = c * a - sn * b;
        sA[i * m + q] = sn * a + c * b;
        const double za = sZ[i * m + p], zb = sZ[i * m + q];
        sZ[i * m + p] = c * za - sn * zb;
        sZ[i * m + q] = sn * za + c * zb;
      }
      __syncthreads();
    }
  }
  if (tid < m) sE[tid] = sA[tid * m + tid];
  __syncthreads();
  if (tid < m) {
    const double e = sE[tid];
    int rank = 0;
    for (int j = 0; j < m; ++j) {
      const double f = sE[j];
      rank += (f < e) || (f == e && j < tid);
    }
    s_sel[rank] = tid;
  }
  __syncthreads();
  // Y = D L^-T Z[:, sel]  (m x B)
  double *Y = coef + size_t(d) * m * B;
  for (int idx = tid; idx < m * B; idx += nt) {
    const int i = idx / B, c = idx % B;
    const int zc = s_sel[c];
    double sum = 0.0;
    for (int l = i; l < m; ++l) sum += sT[l * m + i] * sZ[l * m + zc];
    Y[idx] = sD[i] * sum;
  }
  if (tid < B) th[tid] = sE[s_sel[tid]];
  __syncthreads();
  if (tid == 0) {
    s.has_p = 1;
    s.iters++;
    s.iters_phase++;
    if (prm.phase32) s.iters32++;
    s.have_res = 1;
  }
}

// ---------------------------------------------------------------------------
// Update: X = S Y, P = [W P] Y_wp, HX/HP/MX/MP likewise; W = HX - MX Theta
// ---------------------------------------------------------------------------

template <int B> struct UpdCfg {
  static constexpr int R = 256 / B;      // rows per tile
  static constexpr int THREADS = R * B;
};

template <typename TV, int B>
__global__ void __launch_bounds__(UpdCfg<B>::THREADS)
update_kernel(const Chunk *chunks, const DotState *st, const double *coef, const double *theta,
              TV *X, TV *W, TV *P, TV *HX, TV *HW, TV *HP, TV *MX, TV *MW, TV *MP,
              double *norms) {
  constexpr int m = 3 * B, R = UpdCfg<B>::R;
  using ACC = TV;   // FP32 arithmetic in the FP32 phase, FP64 in the FP64 phase
  __shared__ ACC sY[m * B];
  __shared__ ACC sTh[B];
  __shared__ TV sIn[R * 9 * B];
  __shared__ double sRed[R * B * 2];
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].active) return;
  const int tid = threadIdx.x;
  const double *Yg = coef + size_t(ch.dot) * m * B;
  for (int i = tid; i < m * B; i += blockDim.x) sY[i] = ACC(Yg[i]);
  if (tid < B) sTh[tid] = ACC(theta[size_t(ch.dot) * B + tid]);
  TV *src[9] = {X, W, P, HX, HW, HP, MX, MW, MP};
  const int row = tid / B, j = tid % B;
  double rr = 0.0, mm = 0.0;
  for (int r0 = ch.begin; r0 < ch.end; r0 += R) {
    const int nr = min(R, ch.end - r0);
    __syncthreads();
    for (int idx = tid; idx < 9 * R * B; idx += blockDim.x) {
      const int a = idx / (R * B), rem = idx % (R * B);
      const int rr_ = rem / B, cc = rem % B;
      sIn[rr_ * 9 * B + a * B + cc] = (rr_ < nr) ? src[a][size_t(r0 + rr_) * B + cc] : TV(0);
    }
    __syncthreads();
    if (row < nr) {
      const TV *in = sIn + row * 9 * B;
      ACC x = 0, p = 0, hx = 0, hp = 0, mx = 0, mp = 0;
#pragma unroll
      for (int i = 0; i < B; ++i) {
        const ACC y = sY[i * B + j];
        x = fma(ACC(in[i]), y, x);
        hx = fma(ACC(in[3 * B + i]), y, hx);
        mx = fma(ACC(in[6 * B + i]), y, mx);
      }
#pragma unroll
      for (int i = B; i < 3 * B; ++i) {
        const ACC y = sY[i * B + j];
        const ACC s0 = ACC(in[i]), h0 = ACC(in[3 * B + i]), m0 = ACC(in[6 * B + i]);
        x = fma(s0, y, x);
        hx = fma(h0, y, hx);
        mx = fma(m0, y, mx);
        p = fma(s0, y, p);
        hp = fma(h0, y, hp);
        mp = fma(m0, y, mp);
      }
      const ACC res = hx - sTh[j] * mx;
      const size_t o = size_t(r0 + row) * B + j;
      X[o] = TV(x);
      P[o] = TV(p);
      HX[o] = TV(hx);
      HP[o] = TV(hp);
      MX[o] = TV(mx);
      MP[o] = TV(mp);
      W[o] = TV(res);
      rr += double(res) * double(res);
      mm += double(mx) * double(mx);
    }
  }
  sRed[tid] = rr;
  sRed[R * B + tid] = mm;
  __syncthreads();
  if (tid < B) {
    double a = 0.0, b = 0.0;
    for (int rr_ = 0; rr_ < R; ++rr_) {
      a += sRed[rr_ * B + tid];
      b += sRed[R * B + rr_ * B + tid];
    }
    norms[size_t(blockIdx.x) * 2 * B + tid] = a;
    norms[size_t(blockIdx.x) * 2 * B + B + tid] = b;
  }
}

__global__ void count_active_kernel(const DotState *st, int n, int *out) {
  __shared__ int s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) c += st[i].active;
  atomicAdd(&s, c);
  __syncthreads();
  if (threadIdx.x == 0) *out = s;
}

__global__ void phase_reset_kernel(DotState *st, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  DotState &s = st[i];
  s.active = (s.status != 2) ? 1 : 0;
  s.has_p = 0;
  s.have_res = 0;
  s.iters_phase = 0;
  s.stag = 0;
  s.best = 1e300;
}

template <int B>
__global__ void output_kernel(const Chunk *chunks, const double *X, int k, double *Xout) {
  const Chunk ch = chunks[blockIdx.x];
  for (int idx = threadIdx.x; idx < (ch.end - ch.begin) * k; idx += blockDim.x) {
    const int r = ch.begin + idx / k, j = idx % k;
    Xout[size_t(r) * k + j] = X[size_t(r) * B + j];
  }
}

template <int B>
__global__ void finalize_kernel(const DotState *st, int n, int k, const double *theta,
                                const double *relres, double *E, double *res, int32_t *iters) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n) return;
  for (int j = 0; j < k; ++j) {
    E[size_t(d) * k + j] = theta[size_t(d) * B + j];
    res[size_t(d) * k + j] = relres[size_t(d) * B + j];
  }
  iters[d] = st[d].iters;
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------

struct Layout {
  Chunk *chunks;
  int32_t *row_off;
  DotState *st;
  double *theta, *coef, *relres, *partial, *norms;
  int *count;
  double *slot[9];
  int nchunks;
};

size_t rr_smem_bytes(int B) {
  const int m = 3 * B;
  return size_t(4 * m * m + 2 * m + B) * sizeof(double);
}

int carve(qd::Arena &ar, int n_dots, int64_t n_rows, int B, int nchunks, Layout &L) {
  const int m = 3 * B;
  L.chunks = ar.take<Chunk>(nchunks);
  L.row_off = ar.take<int32_t>(n_dots + 1);
  L.st = ar.take<DotState>(n_dots);
  L.theta = ar.take<double>(size_t(n_dots) * B);
  L.coef = ar.take<double>(size_t(n_dots) * m * B);
  L.relres = ar.take<double>(size_t(n_dots) * B);
  L.partial = ar.take<double>(size_t(nchunks) * 2 * m * m);
  L.norms = ar.take<double>(size_t(nchunks) * 2 * B);
  L.count = ar.take<int>(4);
  for (int i = 0; i < 9; ++i) L.slot[i] = ar.take<double>(size_t(n_rows) * B);
  L.nchunks = nchunks;
  return QD_OK;
}

int count_chunks(int n_dots, const int32_t *row_off) {
  int64_t c = 0;
  for (int d = 0; d < n_dots; ++d) {
    const int n = row_off[d + 1] - row_off[d];
    c += (n + kChunkRows - 1) / kChunkRows;
  }
  return int(c);
}

template <typename TV, int B>
struct Bufs {
  TV *X, *W, *P, *HX, *HW, *HP, *MX, *MW, *MP;
  explicit Bufs(double *const *slot, const int *perm) {
    TV **dst[9] = {&X, &W, &P, &HX, &HW, &HP, &MX, &MW, &MP};
    for (int i = 0; i < 9; ++i) *dst[i] = reinterpret_cast<TV *>(slot[perm[i]]);
  }
};

template <typename TV, int B>
int run_phase(const Layout &L, const int *perm, int n_dots, const int32_t *rowptr,
              const int32_t *col, const double *H, const double *M, const RRParams &prm,
              cudaStream_t s, int &iters_run) {
  Bufs<TV, B> b(L.slot, perm);
  constexpr int G = B / 4;
  const int spmm_threads = 64 * G;
  using GC = GramCfg<B>;
  const size_t rr_smem = rr_smem_bytes(B);
  QD_CUDA_TRY(cudaFuncSetAttribute(rr_kernel<B>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(rr_smem)));
  const int refresh = prm.phase32 ? kRefresh32 : kRefresh64;
  spmm_chunk_kernel<TV, B><<<L.nchunks, spmm_threads, 0, s>>>(L.chunks, L.st, rowptr, col, H, M,
                                                              b.X, b.HX, b.MX);
  QD_CHECK_LAUNCH();
  int host_count = n_dots;
  iters_run = 0;
  for (int it = 0; it < prm.max_iter + 1; ++it) {
    if (it > 0 && it % refresh == 0) {
      spmm_chunk_kernel<TV, B><<<L.nchunks, spmm_threads, 0, s>>>(L.chunks, L.st, rowptr, col,
                                                                  H, M, b.X, b.HX, b.MX);
      QD_CHECK_LAUNCH();
      spmm_chunk_kernel<TV, B><<<L.nchunks, spmm_threads, 0, s>>>(L.chunks, L.st, rowptr, col,
                                                                  H, M, b.P, b.HP, b.MP);
      QD_CHECK_LAUNCH();
    }
    gram_kernel<TV, B><<<L.nchunks, GC::THREADS, 0, s>>>(L.chunks, L.st, b.X, b.W, b.P, b.HX,
                                                         b.HW, b.HP, b.MX, b.MW, b.MP,
                                                         L.partial);
    QD_CHECK_LAUNCH();
    rr_kernel<B><<<n_dots, 256, rr_smem, s>>>(L.st, L.partial, L.norms, L.theta, L.coef,
                                              L.relres, prm);
    QD_CHECK_LAUNCH();
    update_kernel<TV, B><<<L.nchunks, UpdCfg<B>::THREADS, 0, s>>>(
        L.chunks, L.st, L.coef, L.theta, b.X, b.W, b.P, b.HX, b.HW, b.HP, b.MX, b.MW, b.MP,
        L.norms);
    QD_CHECK_LAUNCH();
    spmm_chunk_kernel<TV, B><<<L.nchunks, spmm_threads, 0, s>>>(L.chunks, L.st, rowptr, col, H,
                                                                M, b.W, b.HW, b.MW);
    QD_CHECK_LAUNCH();
    ++iters_run;
    if (it % 8 == 7 || it == prm.max_iter) {
      count_active_kernel<<<1, 256, 0, s>>>(L.st, n_dots, L.count);
      QD_CHECK_LAUNCH();
      QD_CUDA_TRY(cudaMemcpyAsync(&host_count, L.count, sizeof(int), cudaMemcpyDeviceToHost, s));
      QD_CUDA_TRY(cudaStreamSynchronize(s));
      if (host_count == 0) break;
    }
  }
  return QD_OK;
}

template <int B>
int solve_b(int32_t n_dots, const int32_t *h_row_off, const int32_t *d_rowptr,
            const int32_t *d_col, const double *d_H, const double *d_M, int k, int prec_mode,
            double tol, int max_iter, uint64_t seed, double *d_X_out, double *d_E_out,
            double *d_res_out, int32_t *d_iters_out, int32_t *h_info, void *d_work,
            size_t work_bytes, cudaStream_t s) {
  const int64_t n_rows = h_row_off[n_dots];
  const int nchunks = count_chunks(n_dots, h_row_off);
  {
    qd::Arena need(nullptr, 0);
    Layout tmp;
    carve(need, n_dots, n_rows, B, nchunks, tmp);
    if (need.used > work_bytes) return QD_ERR_WORKSPACE;
  }
  if (reinterpret_cast<uintptr_t>(d_work) % 256 != 0) return QD_ERR_WORKSPACE;
  qd::Arena ar(d_work, work_bytes);
  Layout L;
  carve(ar, n_dots, n_rows, B, nchunks, L);
  // chunk table and per-dot state
  std::vector<Chunk> chunks;
  chunks.reserve(nchunks);
  std::vector<DotState> st(n_dots);
  for (int d = 0; d < n_dots; ++d) {
    DotState &x = st[d];
    std::memset(&x, 0, sizeof(x));
    x.active = 1;
    x.best = 1e300;
    x.chunk0 = int(chunks.size());
    for (int r = h_row_off[d]; r < h_row_off[d + 1]; r += kChunkRows)
      chunks.push_back(Chunk{d, r, std::min(r + kChunkRows, h_row_off[d + 1]), 0});
    x.chunk1 = int(chunks.size());
    if (x.chunk1 == x.chunk0) {
      x.active = 0;
      x.status = 2;
    }
  }
  QD_CUDA_TRY(cudaMemcpyAsync(L.chunks, chunks.data(), chunks.size() * sizeof(Chunk),
                              cudaMemcpyHostToDevice, s));
  QD_CUDA_TRY(cudaMemcpyAsync(L.st, st.data(), st.size() * sizeof(DotState),
                              cudaMemcpyHostToDevice, s));
  QD_CUDA_TRY(cudaMemcpyAsync(L.row_off, h_row_off, sizeof(int32_t) * (n_dots + 1),
                              cudaMemcpyHostToDevice, s));
  QD_CUDA_TRY(cudaMemsetAsync(L.theta, 0, sizeof(double) * size_t(n_dots) * B, s));
  QD_CUDA_TRY(cudaMemsetAsync(L.relres, 0, sizeof(double) * size_t(n_dots) * B, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));   // host staging vectors die at return

  const int perm0[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
  int it32 = 0, it64 = 0;
  RRParams prm;
  prm.k = k;
  prm.max_iter = max_iter;
  if (prec_mode == QD_PREC_MIXED) {
    Bufs<float, B> b(L.slot, perm0);
    init_kernel<float, B><<<nchunks, 256, 0, s>>>(L.chunks, L.row_off, seed, b.X, b.W, b.P,
                                                  b.HW, b.MW, b.HP, b.MP);
    QD_CHECK_LAUNCH();
    prm.phase32 = 1;
    prm.tol = std::max(tol, kTol32);
    int st32 = run_phase<float, B>(L, perm0, n_dots, d_rowptr, d_col, d_H, d_M, prm, s, it32);
    if (st32 != QD_OK) return st32;
    // X (float, slot 0) -> double in slot 1; slot 1 becomes X, slot 0 becomes W
    convert_kernel<B><<<nchunks, 256, 0, s>>>(L.chunks, reinterpret_cast<const float *>(L.slot[0]),
                                              L.slot[1]);
    QD_CHECK_LAUNCH();
    const int perm1[9] = {1, 0, 2, 3, 4, 5, 6, 7, 8};
    Bufs<double, B> b64(L.slot, perm1);
    zero_aux_kernel<double, B><<<nchunks, 256, 0, s>>>(L.chunks, b64.W, b64.P, b64.HW, b64.MW,
                                                       b64.HP, b64.MP);
    QD_CHECK_LAUNCH();
    phase_reset_kernel<<<(n_dots + 127) / 128, 128, 0, s>>>(L.st, n_dots);
    QD_CHECK_LAUNCH();
    prm.phase32 = 0;
    prm.tol = tol;
    int st64 = run_phase<double, B>(L, perm1, n_dots, d_rowptr, d_col, d_H, d_M, prm, s, it64);
    if (st64 != QD_OK) return st64;
    output_kernel<B><<<nchunks, 256, 0, s>>>(L.chunks, L.slot[1], k, d_X_out);
    QD_CHECK_LAUNCH();
  } else {
    Bufs<double, B> b(L.slot, perm0);
    init_kernel<double, B><<<nchunks, 256, 0, s>>>(L.chunks, L.row_off, seed, b.X, b.W, b.P,
                                                   b.HW, b.MW, b.HP, b.MP);
    QD_CHECK_LAUNCH();
    prm.phase32 = 0;
    prm.tol = tol;
    int st64 = run_phase<double, B>(L, perm0, n_dots, d_rowptr, d_col, d_H, d_M, prm, s, it64);
    if (st64 != QD_OK) return st64;
    output_kernel<B><<<nchunks, 256, 0, s>>>(L.chunks, L.slot[0], k, d_X_out);
    QD_CHECK_LAUNCH();
  }
  finalize_kernel<B><<<(n_dots + 127) / 128, 128, 0, s>>>(L.st, n_dots, k, L.theta, L.relres,
                                                          d_E_out, d_res_out, d_iters_out);
  QD_CHECK_LAUNCH();
  QD_CUDA_TRY(cudaMemcpyAsync(st.data(), L.st, st.size() * sizeof(DotState),
                              cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  int nconv = 0, nbreak = 0;
  for (auto &x : st) {
    nconv += (x.status == 1);
    nbreak += (x.status == 2);
  }
  if (h_info) {
    h_info[0] = it32 + it64;
    h_info[1] = it32;
    h_info[2] = it64;
    h_info[3] = nconv;
  }
  if (nbreak) return QD_ERR_BREAKDOWN;
  if (nconv != n_dots) return QD_ERR_NOT_CONVERGED;
  return QD_OK;
}

}  // namespace

extern "C" int qd_lobpcg_workspace_size(int32_t n_dots, int64_t n_rows_total, int b,
                                        int prec_mode, size_t *bytes) {
  (void)prec_mode;
  if (!bytes || n_dots <= 0 || n_rows_total <= 0 || b < 4 || b > kMaxB || b % 4) return QD_ERR_INVALID;
  // upper bound on the chunk count: every dot contributes at most one partial chunk
  const int nchunks = int(n_rows_total / kChunkRows) + n_dots;
  qd::Arena ar(nullptr, 0);
  Layout L;
  carve(ar, n_dots, n_rows_total, b, nchunks, L);
  *bytes = ar.used;
  return QD_OK;
}

extern "C" int qd_lobpcg_solve(int32_t n_dots, const int32_t *h_row_off,
                               const int32_t *d_row_off, const int32_t *d_rowptr,
                               const int32_t *d_col, const double *d_H, const double *d_M, int k,
                               int b, int prec_mode, double tol, int max_iter, uint64_t seed,
                               double *d_X_out, double *d_E_out, double *d_res_out,
                               int32_t *d_iters_out, int32_t *h_info, void *d_work,
                               size_t work_bytes, void *stream) {
  (void)d_row_off;
  if (n_dots <= 0 || !h_row_off || !d_rowptr || !d_col || !d_H || !d_M || !d_X_out ||
      !d_E_out || !d_res_out || !d_iters_out || !d_work)
    return QD_ERR_INVALID;
  if (k < 1 || k > b || b < 4 || b > kMaxB || b % 4 != 0) return QD_ERR_INVALID;
  if (prec_mode != QD_PREC_FP64 && prec_mode != QD_PREC_MIXED) return QD_ERR_INVALID;
  if (!(tol > 0.0) || max_iter < 1) return QD_ERR_INVALID;
  for (int d = 0; d < n_dots; ++d)
    if (h_row_off[d + 1] < h_row_off[d]) return QD_ERR_INVALID;
  if (h_row_off[0] != 0) return QD_ERR_INVALID;
  for (int d = 0; d < n_dots; ++d)
    if (h_row_off[d + 1] - h_row_off[d] < b + 1) return QD_ERR_INVALID;  // need n > b
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (b) {
    case 4: return solve_b<4>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, d_work, work_bytes, s);
    case 8: return solve_b<8>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, d_work, work_bytes, s);
    case 12: return solve_b<12>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, d_work, work_bytes, s);
    default: return solve_b<16>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, d_work, work_bytes, s);
  }
}

// Single dual SpMM (one problem, all rows).
template <typename TV, int B>
__global__ void spmm_plain_kernel(int32_t n, const int32_t *rowptr, const int32_t *col,
                                  const double *H, const double *M, const TV *X, TV *HX, TV *MX) {
  constexpr int G = B / 4;
  const int sub = threadIdx.x / G, g = threadIdx.x % G;
  const int rpb = blockDim.x / G;
  for (int r = blockIdx.x * rpb + sub; r < n; r += gridDim.x * rpb) {
    if (M && MX)
      qd::spmm_row<TV, B, true>(r, g, rowptr, col, H, M, X, HX, MX);
    else
      qd::spmm_row<TV, B, false>(r, g, rowptr, col, H, nullptr, X, HX, nullptr);
  }
}

template <typename TV, int B>
static int spmm_plain(int32_t n, const int32_t *rowptr, const int32_t *col, const double *H,
                      const double *M, const void *X, void *HX, void *MX, cudaStream_t s) {
  constexpr int G = B / 4;
  const int threads = 64 * G;
  int64_t blocks = (int64_t(n) + 63) / 64;
  if (blocks > 148 * 32) blocks = 148 * 32;
  spmm_plain_kernel<TV, B><<<int(blocks), threads, 0, s>>>(
      n, rowptr, col, H, M, static_cast<const TV *>(X), static_cast<TV *>(HX),
      static_cast<TV *>(MX));
  QD_CHECK_LAUNCH();
  return QD_OK;
}

extern "C" int qd_spmm_dual(int32_t n_rows, int b, int vec_fp32, const int32_t *d_rowptr,
                            const int32_t *d_col, const double *d_H, const double *d_M,
                            const void *d_X, void *d_HX, void *d_MX, void *stream) {
  if (n_rows < 0 || !d_rowptr || !d_col || !d_H || !d_X || !d_HX) return QD_ERR_INVALID;
  if ((d_M == nullptr) != (d_MX == nullptr)) return QD_ERR_INVALID;
  if (n_rows == 0) return QD_OK;
  const int align = vec_fp32 ? 16 : 16;
  if (reinterpret_cast<uintptr_t>(d_X) % align || reinterpret_cast<uintptr_t>(d_HX) % align ||
      (d_MX && reinterpret_cast<uintptr_t>(d_MX) % align))
    return QD_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define QD_SPMM_CASE(BB)                                                                   \
  case BB:                                                                                 \
    return vec_fp32 ? spmm_plain<float, BB>(n_rows, d_rowptr, d_col, d_H, d_M, d_X, d_HX,   \
                                            d_MX, s)                                       \
                    : spmm_plain<double, BB>(n_rows, d_rowptr, d_col, d_H, d_M, d_X, d_HX,  \
                                             d_MX, s);
  switch (b) {
    QD_SPMM_CASE(4)
    QD_SPMM_CASE(8)
    QD_SPMM_CASE(12)
    QD_SPMM_CASE(16)
    default: return QD_ERR_INVALID;
  }
#undef QD_SPMM_CASE
}
