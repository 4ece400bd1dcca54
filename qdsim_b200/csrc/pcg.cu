// Jacobi-preconditioned conjugate gradients, FP64, for nrhs right-hand sides
// sharing one SPD matrix (Poisson step of the self-consistent loop).
//
// Replaces PoissonSolver::solve (backend/src/poisson.cpp:320-334,
// SimplicialLDLT) and the spsolve / cg calls of CythonPoissonSolver.solve
// (qdsim_cython/solvers/poisson_solver.pyx:238-247).  Dirichlet rows are kept
// at their input value and eliminated from the iteration (the reference
// replaces those rows by identity rows, :276-308, which gives the same
// solution on the free rows).
//
// Vectors are row-major (x[row*nrhs + j]).  Every thread owns one fixed
// column j = tid % nrhs for the whole launch (block size and grid stride are
// multiples of nrhs) and steps over rows, so the per-column dot products
// reduce in a fixed order: bitwise reproducible, no atomics on values.
//
// One iteration is two launches.  (1) p = z + beta p_prev fused into
// Ap = A p: every gathered neighbour value is recomputed as
// fma(beta, p_prev, z), the same expression the row's owner stores, so the
// product sees exactly the stored direction (p alternates between two
// buffers).  (2) x += alpha p, r -= alpha Ap, z = D^-1 r.  Each launch leaves
// per-block column partials; the block that finishes last (block counter)
// sums them in block order and computes the step scalars, so no separate
// reduction launch sits between the two.  The host reads only the
// convergence flag, every 16 iterations.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>
#include "common.h"

namespace {

constexpr int kMaxRhs = 256;
constexpr int kThreads = 1024;     // per block, rounded down to a multiple of nrhs
constexpr int kGridBlocks = 2 * 148;   // two blocks per SM of a B200 (32 registers)

struct Cfg {
  int n, nrhs, threads, blocks;
};

// partials: part[(kind * nrhs + j) * blocks + block]; kinds 0 r.z, 1 r.r, 2 p.Ap
// step scalars per column: sc[j * 5 + {0 rz, 1 rr0, 2 alpha, 3 beta, 4 rr}]

// Column sums of this block's per-thread values v0 (and v1 when NV == 2) into
// part[k0] (and part[k0 + 1]): threads t, t + nrhs, ... in order.
template <int NV>
__device__ inline void block_col_reduce(double v0, double v1, double *red, const Cfg &c,
                                        double *part_k0) {
  red[threadIdx.x] = v0;
  if (NV == 2) red[blockDim.x + threadIdx.x] = v1;
  __syncthreads();
  if (threadIdx.x < c.nrhs) {
    double s0 = 0.0, s1 = 0.0;
    for (int t = threadIdx.x; t < blockDim.x; t += c.nrhs) {
      s0 += red[t];
      if (NV == 2) s1 += red[blockDim.x + t];
    }
    part_k0[size_t(threadIdx.x) * c.blocks + blockIdx.x] = s0;
    if (NV == 2) part_k0[size_t(c.nrhs + threadIdx.x) * c.blocks + blockIdx.x] = s1;
  }
  __syncthreads();
}

// True in every thread of the block that finished last; that block then sees
// every other block's partials.  The barrier orders this block's partial
// writes before thread 0's fence, which makes them visible device-wide
// before the counter moves.
__device__ inline bool last_block(unsigned *counter) {
  __shared__ unsigned s_last;
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// Step scalars in the last block.  mode 0: initial (rz, rr0, done); mode 1:
// alpha = rz / pAp (0 for a converged column); mode 2: beta, rr, done.
// Column j = threadIdx.x / L is summed by L = blockDim / nrhs lanes: lane l
// takes blocks l, l + L, ... in order (kU loads of each kind in flight), then
// the lane sums are added in lane order.
constexpr int kU = 4;

__device__ void finish_scalars(int mode, const Cfg &c, const double *part, double *sc, int *done,
                               unsigned *counter, double tol, double *red) {
  __shared__ int s_all;
  if (threadIdx.x == 0) s_all = 1;
  const int L = blockDim.x / c.nrhs;
  const int j = threadIdx.x / L, l = threadIdx.x % L;
  const bool two = mode != 1;
  const double *pa = part + (size_t(mode == 1 ? 2 : 0) * c.nrhs + j) * c.blocks;
  const double *pb = part + (size_t(c.nrhs) + j) * c.blocks;
  double a = 0.0, b = 0.0;
  for (int b0 = l; b0 < c.blocks; b0 += kU * L) {
    double va[kU], vb[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int k = b0 + u * L;
      va[u] = k < c.blocks ? __ldcg(pa + k) : 0.0;
      vb[u] = (two && k < c.blocks) ? __ldcg(pb + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      a += va[u];
      b += vb[u];
    }
  }
  red[threadIdx.x] = a;
  red[blockDim.x + threadIdx.x] = b;
  __syncthreads();
  double sa = 0.0, sb = 0.0;
  if (l == 0)
    for (int q = 0; q < L; ++q) {
      sa += red[threadIdx.x + q];
      sb += red[blockDim.x + threadIdx.x + q];
    }
  // mode 0: the reference residual ||b - A x_D||^2 (kind 2), x_D = the
  // initial x with its free entries zeroed (the Dirichlet values alone)
  double sref = 0.0;
  if (mode == 0) {
    __syncthreads();
    const double *pc = part + (size_t(2) * c.nrhs + j) * c.blocks;
    double cz = 0.0;
    for (int k = l; k < c.blocks; k += L) cz += __ldcg(pc + k);
    red[threadIdx.x] = cz;
    __syncthreads();
    if (l == 0)
      for (int q = 0; q < L; ++q) sref += red[threadIdx.x + q];
  }
  if (l == 0) {
    double *s = sc + size_t(j) * 5;
    if (mode == 0) {
      // relative to the zero-guess residual, so that a warm start does not
      // tighten the target (the initial residual when that one is zero)
      const double ref = sref > 0.0 ? sref : sb;
      s[0] = sa;
      s[1] = ref;
      s[2] = 0.0;
      s[3] = 0.0;
      s[4] = sb;
      if (!(sb <= tol * tol * ref)) atomicAnd(&s_all, 0);
    } else if (mode == 1) {
      s[2] = (sa > 0.0 && s[4] > tol * tol * s[1]) ? s[0] / sa : 0.0;
    } else {
      s[3] = (s[0] > 0.0) ? sa / s[0] : 0.0;
      s[0] = sa;
      s[4] = sb;
      if (!(sb <= tol * tol * s[1])) atomicAnd(&s_all, 0);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (mode != 1) *done = s_all;
    *counter = 0u;
  }
}

// r = b - A x (free rows), z = D^-1 r, p_prev = 0; partials r.z, r.r and
// |b - A x_D|^2 (x_D: x with its free entries zeroed)
__global__ void __launch_bounds__(kThreads, 2)
pcg_init_kernel(Cfg c, const int32_t *rowptr, const int32_t *col, const double *A,
                const double *Bv, const double *X, const int32_t *fixed, double *R, double *Z,
                double *P, double *dinv, double *part, double *sc, int *done, unsigned *counter,
                double tol) {
  extern __shared__ double red[];
  const int j = threadIdx.x % c.nrhs, rpb = blockDim.x / c.nrhs;
  const int step = gridDim.x * rpb;
  double rz = 0.0, rr = 0.0, rr0 = 0.0;
  for (int row = blockIdx.x * rpb + threadIdx.x / c.nrhs; row < c.n; row += step) {
    const size_t idx = size_t(row) * c.nrhs + j;
    double r = 0.0, r0 = 0.0, di = 0.0;
    if (!fixed || !fixed[row]) {
      double ax = 0.0, axd = 0.0, diag = 0.0;
      for (int p = rowptr[row]; p < rowptr[row + 1]; ++p) {
        const int cj = col[p];
        const double a = A[p], xv = X[size_t(cj) * c.nrhs + j];
        ax = fma(a, xv, ax);
        if (fixed && fixed[cj]) axd = fma(a, xv, axd);
        if (cj == row) diag = a;
      }
      r = Bv[idx] - ax;
      r0 = Bv[idx] - axd;
      di = diag != 0.0 ? 1.0 / diag : 0.0;
    }
    if (j == 0) dinv[row] = di;
    const double z = r * di;
    R[idx] = r;
    Z[idx] = z;
    P[idx] = 0.0;
    rz += r * z;
    rr += r * r;
    rr0 += r0 * r0;
  }
  block_col_reduce<2>(rz, rr, red, c, part);
  block_col_reduce<1>(rr0, 0.0, red, c, part + size_t(2) * c.nrhs * c.blocks);
  if (last_block(counter)) finish_scalars(0, c, part, sc, done, counter, tol, red);
}

// p = z + beta p_prev, Ap = A p (free rows; p is zero on fixed rows); partial p.Ap
__global__ void __launch_bounds__(kThreads, 2)
pcg_spmv_kernel(Cfg c, const int32_t *rowptr, const int32_t *col, const double *A,
                const int32_t *fixed, const double *Z, const double *Pprev, double *P, double *AP,
                double *part, double *sc, int *done, unsigned *counter, double tol) {
  extern __shared__ double red[];
  if (*done) return;
  const int j = threadIdx.x % c.nrhs, rpb = blockDim.x / c.nrhs;
  const int step = gridDim.x * rpb;
  const double beta = sc[size_t(j) * 5 + 3];
  double pap = 0.0;
  for (int row = blockIdx.x * rpb + threadIdx.x / c.nrhs; row < c.n; row += step) {
    const size_t idx = size_t(row) * c.nrhs + j;
    double ap = 0.0;
    if (!fixed || !fixed[row]) {
      for (int p = rowptr[row]; p < rowptr[row + 1]; ++p) {
        const size_t q = size_t(col[p]) * c.nrhs + j;
        ap = fma(A[p], fma(beta, Pprev[q], Z[q]), ap);
      }
    }
    const double pi = fma(beta, Pprev[idx], Z[idx]);
    P[idx] = pi;
    AP[idx] = ap;
    pap += pi * ap;
  }
  block_col_reduce<1>(pap, 0.0, red, c, part + size_t(2) * c.nrhs * c.blocks);
  if (last_block(counter)) finish_scalars(1, c, part, sc, done, counter, tol, red);
}

// x += alpha p, r -= alpha Ap, z = D^-1 r; partials r.z, r.r
__global__ void __launch_bounds__(kThreads, 2)
pcg_axpy_kernel(Cfg c, const double *dinv, double *X, double *R, double *Z, const double *P,
                const double *AP, double *part, double *sc, int *done, unsigned *counter,
                double tol) {
  extern __shared__ double red[];
  if (*done) return;
  const int j = threadIdx.x % c.nrhs, rpb = blockDim.x / c.nrhs;
  const int step = gridDim.x * rpb;
  const double alpha = sc[size_t(j) * 5 + 2];
  double rz = 0.0, rr = 0.0;
  for (int row = blockIdx.x * rpb + threadIdx.x / c.nrhs; row < c.n; row += step) {
    const size_t idx = size_t(row) * c.nrhs + j;
    X[idx] = fma(alpha, P[idx], X[idx]);
    const double r = fma(-alpha, AP[idx], R[idx]);
    const double z = r * dinv[row];
    R[idx] = r;
    Z[idx] = z;
    rz += r * z;
    rr += r * r;
  }
  block_col_reduce<2>(rz, rr, red, c, part);
  if (last_block(counter)) finish_scalars(2, c, part, sc, done, counter, tol, red);
}

Cfg make_cfg(int n, int nrhs) {
  Cfg c;
  c.n = n;
  c.nrhs = nrhs;
  c.threads = (kThreads / nrhs) * nrhs;
  const int rpb = c.threads / nrhs;
  const int want = (n + rpb - 1) / rpb;
  c.blocks = std::min(std::max(want, 1), kGridBlocks);
  return c;
}

struct PcgLayout {
  double *R, *Z, *P[2], *AP, *dinv, *part, *sc;
  int *done;
  unsigned *counter;
};

void carve(qd::Arena &ar, const Cfg &c, PcgLayout &L) {
  const size_t nv = size_t(c.n) * c.nrhs;
  L.R = ar.take<double>(nv);
  L.Z = ar.take<double>(nv);
  L.P[0] = ar.take<double>(nv);
  L.P[1] = ar.take<double>(nv);
  L.AP = ar.take<double>(nv);
  L.dinv = ar.take<double>(c.n);
  L.part = ar.take<double>(size_t(c.blocks) * 3 * c.nrhs);
  L.sc = ar.take<double>(size_t(c.nrhs) * 5);
  L.done = ar.take<int>(4);
  L.counter = ar.take<unsigned>(4);
}

// The iteration on a carved layout.  The block counter is zeroed first; every
// other scratch word is written before it is read.
int run_pcg(const Cfg &c, const PcgLayout &L, const int32_t *d_rowptr, const int32_t *d_col,
            const double *d_A, const double *d_B, double *d_X, const int32_t *d_fixed,
            double tol, int max_iter, int32_t *h_iters, double *h_relres, cudaStream_t s) {
  const size_t smem = 2 * size_t(c.threads) * sizeof(double);
  QD_CUDA_TRY(cudaMemsetAsync(L.counter, 0, 4 * sizeof(unsigned), s));
  pcg_init_kernel<<<c.blocks, c.threads, smem, s>>>(c, d_rowptr, d_col, d_A, d_B, d_X, d_fixed,
                                                    L.R, L.Z, L.P[0], L.dinv, L.part, L.sc,
                                                    L.done, L.counter, tol);
  QD_CHECK_LAUNCH();
  int it = 0, done = 0;
  const int check = 16;
  for (it = 0; it < max_iter; ++it) {
    const double *Pprev = L.P[it & 1];
    double *P = L.P[(it + 1) & 1];
    pcg_spmv_kernel<<<c.blocks, c.threads, smem, s>>>(c, d_rowptr, d_col, d_A, d_fixed, L.Z,
                                                      Pprev, P, L.AP, L.part, L.sc, L.done,
                                                      L.counter, tol);
    QD_CHECK_LAUNCH();
    pcg_axpy_kernel<<<c.blocks, c.threads, smem, s>>>(c, L.dinv, d_X, L.R, L.Z, P, L.AP, L.part,
                                                      L.sc, L.done, L.counter, tol);
    QD_CHECK_LAUNCH();
    if ((it + 1) % check == 0 || it + 1 == max_iter) {
      QD_CUDA_TRY(cudaMemcpyAsync(&done, L.done, sizeof(int), cudaMemcpyDeviceToHost, s));
      QD_CUDA_TRY(cudaStreamSynchronize(s));
      if (done) {
        ++it;
        break;
      }
    }
  }
  double sc[kMaxRhs * 5];
  QD_CUDA_TRY(cudaMemcpyAsync(sc, L.sc, size_t(c.nrhs) * 5 * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaMemcpyAsync(&done, L.done, sizeof(int), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  double worst = 0.0;
  for (int j = 0; j < c.nrhs; ++j) {
    const double rr0 = sc[size_t(j) * 5 + 1], rr = sc[size_t(j) * 5 + 4];
    worst = std::max(worst, rr0 > 0.0 ? std::sqrt(rr / rr0) : 0.0);
  }
  if (h_iters) *h_iters = it;
  if (h_relres) *h_relres = worst;
  return done ? QD_OK : QD_ERR_NOT_CONVERGED;
}

}  // namespace

extern "C" int qd_pcg_workspace_size(int32_t n, int nrhs, size_t *bytes) {
  if (!bytes || n <= 0 || nrhs < 1 || nrhs > kMaxRhs) return QD_ERR_INVALID;
  Cfg c = make_cfg(n, nrhs);
  qd::Arena ar(nullptr, 0);
  PcgLayout L;
  carve(ar, c, L);
  *bytes = ar.used;
  return QD_OK;
}

extern "C" int qd_pcg_solve(int32_t n, int nrhs, const int32_t *d_rowptr, const int32_t *d_col,
                            const double *d_A, const double *d_B, double *d_X,
                            const int32_t *d_fixed, double tol, int max_iter, int32_t *h_iters,
                            double *h_relres, void *d_work, size_t work_bytes, void *stream) {
  if (n <= 0 || nrhs < 1 || nrhs > kMaxRhs || !d_rowptr || !d_col || !d_A || !d_B || !d_X ||
      !d_work || !(tol > 0.0) || max_iter < 1)
    return QD_ERR_INVALID;
  Cfg c = make_cfg(n, nrhs);
  {
    qd::Arena need(nullptr, 0);
    PcgLayout t;
    carve(need, c, t);
    if (need.used > work_bytes) return QD_ERR_WORKSPACE;
  }
  if (reinterpret_cast<uintptr_t>(d_work) % 256 != 0) return QD_ERR_WORKSPACE;
  qd::Arena ar(d_work, work_bytes);
  PcgLayout L;
  carve(ar, c, L);
  return run_pcg(c, L, d_rowptr, d_col, d_A, d_B, d_X, d_fixed, tol, max_iter, h_iters,
                 h_relres, static_cast<cudaStream_t>(stream));
}

// Y = alpha * A X for nrhs row-major columns (generic CSR product, FP64).
__global__ void csr_spmv_multi_kernel(int32_t n, int nrhs, const int32_t *rowptr,
                                      const int32_t *col, const double *A, const double *X,
                                      double *Y, double alpha) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < int64_t(n) * nrhs;
       idx += stride) {
    const int row = int(idx / nrhs), j = int(idx % nrhs);
    double acc = 0.0;
    for (int p = rowptr[row]; p < rowptr[row + 1]; ++p)
      acc = fma(A[p], X[size_t(col[p]) * nrhs + j], acc);
    Y[idx] = alpha * acc;
  }
}

extern "C" int qd_csr_spmv(int32_t n, int nrhs, const int32_t *d_rowptr, const int32_t *d_col,
                           const double *d_A, const double *d_X, double *d_Y, double alpha,
                           void *stream) {
  if (n < 0 || nrhs < 1 || !d_rowptr || !d_col || !d_A || !d_X || !d_Y) return QD_ERR_INVALID;
  if (n == 0) return QD_OK;
  const int64_t total = int64_t(n) * nrhs;
  const int blocks = int(std::min<int64_t>((total + 255) / 256, 148 * 16));
  csr_spmv_multi_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      n, nrhs, d_rowptr, d_col, d_A, d_X, d_Y, alpha);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

// ---------------------------------------------------------------------------
// PCG with library-owned scratch, for callers that cannot allocate device
// memory themselves (see qd_pcg_solve_static in qdsim_b200.h).
// ---------------------------------------------------------------------------

namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;   // 16 MiB per device

// Every GPU that loads the library reserves this array until the process exits.
static __device__ __align__(256) unsigned char g_pcg_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void *g_static_ptr[64] = {nullptr};

// Device address of g_pcg_scratch on the current device.  In host code the
// symbol is only a host-side stand-in, so the address must be looked up with
// cudaGetSymbolAddress, once per device, with that device current.
int static_scratch(void **out) {
  int dev = 0;
  QD_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return QD_ERR_LIMIT;
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[dev]) {
    void *p = nullptr;
    QD_CUDA_TRY(cudaGetSymbolAddress(&p, g_pcg_scratch));
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return QD_OK;
}

}  // namespace

extern "C" size_t qd_pcg_static_scratch_bytes(void) { return kStaticScratchBytes; }

extern "C" int qd_pcg_solve_static(int32_t n, int nrhs, const int32_t *d_rowptr,
                                   const int32_t *d_col, const double *d_A, const double *d_B,
                                   double *d_X, const int32_t *d_fixed, double tol, int max_iter,
                                   int32_t *h_iters, double *h_relres, void *stream) {
  if (n <= 0 || nrhs < 1 || nrhs > kMaxRhs || !d_rowptr || !d_col || !d_A || !d_B || !d_X ||
      !(tol > 0.0) || max_iter < 1)
    return QD_ERR_INVALID;
  Cfg c = make_cfg(n, nrhs);
  {
    qd::Arena need(nullptr, 0);
    PcgLayout t;
    carve(need, c, t);
    if (need.used > kStaticScratchBytes) return QD_ERR_LIMIT;
  }
  void *scratch = nullptr;
  int st = static_scratch(&scratch);
  if (st != QD_OK) return st;
  qd::Arena ar(scratch, kStaticScratchBytes);
  PcgLayout L;
  carve(ar, c, L);
  // The block counter is zeroed at the start of the call and every other
  // scratch word (residual, search directions, partial sums, step scalars,
  // done flag) is written before it is read, so the contents left by an
  // earlier call need no clearing.
  return run_pcg(c, L, d_rowptr, d_col, d_A, d_B, d_X, d_fixed, tol, max_iter, h_iters,
                 h_relres, static_cast<cudaStream_t>(stream));
}
