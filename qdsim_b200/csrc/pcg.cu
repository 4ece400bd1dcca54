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
// multiples of nrhs), so the per-column dot products reduce in a fixed order:
// bitwise reproducible, no atomics.  The step scalars are computed on the
// device; the host only reads the convergence flag every few iterations.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>
#include "common.h"

namespace {

constexpr int kMaxRhs = 256;

struct Cfg {
  int n, nrhs, threads, blocks;
};

__device__ inline void block_col_reduce(double v, double *red, int nrhs, double *out_block) {
  // red: blockDim doubles; threads t and t' share a column iff t % nrhs == t' % nrhs
  red[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < nrhs) {
    double s = 0.0;
    for (int t = threadIdx.x; t < blockDim.x; t += nrhs) s += red[t];
    out_block[threadIdx.x] = s;
  }
  __syncthreads();
}

// r = b - A x (free rows), z = D^-1 r, p = z; partials: r.z and r.r
__global__ void pcg_init_kernel(Cfg c, const int32_t *rowptr, const int32_t *col, const double *A,
                                const double *Bv, const double *X, const int32_t *fixed,
                                double *R, double *Z, double *P, double *dinv, double *part) {
  extern __shared__ double red[];
  const int stride = gridDim.x * blockDim.x;
  double rz = 0.0, rr = 0.0;
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < int64_t(c.n) * c.nrhs;
       idx += stride) {
    const int row = int(idx / c.nrhs), j = int(idx % c.nrhs);
    double r = 0.0, di = 0.0;
    if (!fixed || !fixed[row]) {
      double ax = 0.0, diag = 0.0;
      for (int p = rowptr[row]; p < rowptr[row + 1]; ++p) {
        const int cj = col[p];
        ax = fma(A[p], X[size_t(cj) * c.nrhs + j], ax);
        if (cj == row) diag = A[p];
      }
      r = Bv[idx] - ax;
      di = diag != 0.0 ? 1.0 / diag : 0.0;
    }
    if (j == 0) dinv[row] = di;
    const double z = r * di;
    R[idx] = r;
    Z[idx] = z;
    P[idx] = z;
    rz += r * z;
    rr += r * r;
  }
  block_col_reduce(rz, red, c.nrhs, part + size_t(blockIdx.x) * 3 * c.nrhs);
  block_col_reduce(rr, red, c.nrhs, part + size_t(blockIdx.x) * 3 * c.nrhs + c.nrhs);
}

// Ap = A p (free rows; p is zero on fixed rows); partial p.Ap
__global__ void pcg_spmv_kernel(Cfg c, const int32_t *rowptr, const int32_t *col, const double *A,
                                const int32_t *fixed, const double *P, double *AP,
                                const int *done, double *part) {
  extern __shared__ double red[];
  if (*done) return;
  const int stride = gridDim.x * blockDim.x;
  double pap = 0.0;
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < int64_t(c.n) * c.nrhs;
       idx += stride) {
    const int row = int(idx / c.nrhs), j = int(idx % c.nrhs);
    double ap = 0.0;
    if (!fixed || !fixed[row]) {
      for (int p = rowptr[row]; p < rowptr[row + 1]; ++p)
        ap = fma(A[p], P[size_t(col[p]) * c.nrhs + j], ap);
    }
    AP[idx] = ap;
    pap += P[idx] * ap;
  }
  block_col_reduce(pap, red, c.nrhs, part + size_t(blockIdx.x) * 3 * c.nrhs + 2 * c.nrhs);
}

// scalars: mode 0 -> initial (rz, rr0); mode 1 -> alpha = rz / pAp; mode 2 -> beta, convergence
// The per-block partials of a column are summed by L = kScalarThreads / nrhs
// lanes (lane l takes blocks l, l + L, ...), then the L lane sums in lane
// order: a fixed order, so the result is reproducible.
constexpr int kScalarThreads = 1024;

__global__ void __launch_bounds__(kScalarThreads)
pcg_scalar_kernel(Cfg c, int mode, const double *part, double *sc, int *done, double tol) {
  // sc layout per column: [rz, rr0, alpha, beta, rr]
  __shared__ double s_a[kScalarThreads], s_b[kScalarThreads];
  __shared__ int s_all;
  const int t = threadIdx.x;
  const int L = kScalarThreads / c.nrhs;
  const int j = t / L, l = t % L;
  if (t == 0) s_all = 1;
  // partial kinds: 0 r.z, 1 r.r (modes 0, 2); 2 p.Ap (mode 1)
  const int ka = mode == 1 ? 2 : 0, kb = 1;
  double a = 0.0, b = 0.0;
  if (j < c.nrhs) {
    for (int blk = l; blk < c.blocks; blk += L) {
      a += part[size_t(blk) * 3 * c.nrhs + size_t(ka) * c.nrhs + j];
      if (mode != 1) b += part[size_t(blk) * 3 * c.nrhs + size_t(kb) * c.nrhs + j];
    }
  }
  s_a[t] = a;
  s_b[t] = b;
  __syncthreads();
  if (j < c.nrhs && l == 0) {
    double sa = 0.0, sb = 0.0;
    for (int q = 0; q < L; ++q) {
      sa += s_a[t + q];
      sb += s_b[t + q];
    }
    double *s = sc + size_t(j) * 5;
    if (mode == 0) {
      const double rz = sa, rr = sb;
      s[0] = rz;
      s[1] = rr;
      s[4] = rr;
      if (!(rr > 0.0)) s[2] = 0.0;
      const bool conv = !(rr > 0.0);
      if (!conv) atomicAnd(&s_all, 0);
    } else if (mode == 1) {
      const double pap = sa;
      s[2] = (pap > 0.0 && s[4] > tol * tol * s[1]) ? s[0] / pap : 0.0;
    } else {
      const double rz = sa, rr = sb;
      s[3] = (s[0] > 0.0) ? rz / s[0] : 0.0;
      s[0] = rz;
      s[4] = rr;
      const bool conv = rr <= tol * tol * s[1];
      if (!conv) atomicAnd(&s_all, 0);
    }
  }
  __syncthreads();
  if (t == 0 && mode != 1) *done = s_all;
}

// x += alpha p, r -= alpha Ap, z = D^-1 r; partials r.z, r.r
__global__ void pcg_axpy_kernel(Cfg c, const double *sc, const double *dinv, double *X, double *R,
                                double *Z, const double *P, const double *AP, const int *done,
                                double *part) {
  extern __shared__ double red[];
  if (*done) return;
  const int stride = gridDim.x * blockDim.x;
  double rz = 0.0, rr = 0.0;
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < int64_t(c.n) * c.nrhs;
       idx += stride) {
    const int row = int(idx / c.nrhs), j = int(idx % c.nrhs);
    const double alpha = sc[size_t(j) * 5 + 2];
    X[idx] = fma(alpha, P[idx], X[idx]);
    const double r = fma(-alpha, AP[idx], R[idx]);
    const double z = r * dinv[row];
    R[idx] = r;
    Z[idx] = z;
    rz += r * z;
    rr += r * r;
  }
  block_col_reduce(rz, red, c.nrhs, part + size_t(blockIdx.x) * 3 * c.nrhs);
  block_col_reduce(rr, red, c.nrhs, part + size_t(blockIdx.x) * 3 * c.nrhs + c.nrhs);
}

__global__ void pcg_dir_kernel(Cfg c, const double *sc, const double *Z, double *P, const int *done) {
  if (*done) return;
  const int stride = gridDim.x * blockDim.x;
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < int64_t(c.n) * c.nrhs;
       idx += stride) {
    const int j = int(idx % c.nrhs);
    P[idx] = fma(sc[size_t(j) * 5 + 3], P[idx], Z[idx]);
  }
}

Cfg make_cfg(int n, int nrhs) {
  Cfg c;
  c.n = n;
  c.nrhs = nrhs;
  c.threads = (256 / nrhs) * nrhs;
  int64_t want = (int64_t(n) * nrhs + c.threads - 1) / c.threads;
  c.blocks = int(std::min<int64_t>(std::max<int64_t>(want, 1), 148 * 8));
  return c;
}

struct PcgLayout {
  double *R, *Z, *P, *AP, *dinv, *part, *sc;
  int *done;
};

void carve(qd::Arena &ar, const Cfg &c, PcgLayout &L) {
  const size_t nv = size_t(c.n) * c.nrhs;
  L.R = ar.take<double>(nv);
  L.Z = ar.take<double>(nv);
  L.P = ar.take<double>(nv);
  L.AP = ar.take<double>(nv);
  L.dinv = ar.take<double>(c.n);
  L.part = ar.take<double>(size_t(c.blocks) * 3 * c.nrhs);
  L.sc = ar.take<double>(size_t(c.nrhs) * 5);
  L.done = ar.take<int>(4);
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
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t smem = size_t(c.threads) * sizeof(double);
  pcg_init_kernel<<<c.blocks, c.threads, smem, s>>>(c, d_rowptr, d_col, d_A, d_B, d_X, d_fixed,
                                                    L.R, L.Z, L.P, L.dinv, L.part);
  QD_CHECK_LAUNCH();
  pcg_scalar_kernel<<<1, kScalarThreads, 0, s>>>(c, 0, L.part, L.sc, L.done, tol);
  QD_CHECK_LAUNCH();
  int it = 0, done = 0;
  const int check = 16;
  for (it = 0; it < max_iter; ++it) {
    pcg_spmv_kernel<<<c.blocks, c.threads, smem, s>>>(c, d_rowptr, d_col, d_A, d_fixed, L.P,
                                                      L.AP, L.done, L.part);
    QD_CHECK_LAUNCH();
    pcg_scalar_kernel<<<1, kScalarThreads, 0, s>>>(c, 1, L.part, L.sc, L.done, tol);
    QD_CHECK_LAUNCH();
    pcg_axpy_kernel<<<c.blocks, c.threads, smem, s>>>(c, L.sc, L.dinv, d_X, L.R, L.Z, L.P, L.AP,
                                                      L.done, L.part);
    QD_CHECK_LAUNCH();
    pcg_scalar_kernel<<<1, kScalarThreads, 0, s>>>(c, 2, L.part, L.sc, L.done, tol);
    QD_CHECK_LAUNCH();
    pcg_dir_kernel<<<c.blocks, c.threads, 0, s>>>(c, L.sc, L.Z, L.P, L.done);
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
  std::vector<double> sc(size_t(c.nrhs) * 5);
  QD_CUDA_TRY(cudaMemcpyAsync(sc.data(), L.sc, sc.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaMemcpyAsync(&done, L.done, sizeof(int), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  double worst = 0.0;
  for (int j = 0; j < c.nrhs; ++j) {
    const double rr0 = sc[size_t(j) * 5 + 1], rr = sc[size_t(j) * 5 + 4];
    const double rel = rr0 > 0.0 ? std::sqrt(rr / rr0) : 0.0;
    worst = std::max(worst, rel);
  }
  if (h_iters) *h_iters = it;
  if (h_relres) *h_relres = worst;
  return done ? QD_OK : QD_ERR_NOT_CONVERGED;
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
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t smem = size_t(c.threads) * sizeof(double);
  // Every scratch word (residual, search direction, partial sums, step scalars
  // and the done flag) is written before it is read in this call, so the
  // contents left by an earlier call need no clearing.
  pcg_init_kernel<<<c.blocks, c.threads, smem, s>>>(c, d_rowptr, d_col, d_A, d_B, d_X, d_fixed,
                                                    L.R, L.Z, L.P, L.dinv, L.part);
  QD_CHECK_LAUNCH();
  pcg_scalar_kernel<<<1, kScalarThreads, 0, s>>>(c, 0, L.part, L.sc, L.done, tol);
  QD_CHECK_LAUNCH();
  int it = 0, done = 0;
  for (it = 0; it < max_iter; ++it) {
    pcg_spmv_kernel<<<c.blocks, c.threads, smem, s>>>(c, d_rowptr, d_col, d_A, d_fixed, L.P,
                                                      L.AP, L.done, L.part);
    QD_CHECK_LAUNCH();
    pcg_scalar_kernel<<<1, kScalarThreads, 0, s>>>(c, 1, L.part, L.sc, L.done, tol);
    QD_CHECK_LAUNCH();
    pcg_axpy_kernel<<<c.blocks, c.threads, smem, s>>>(c, L.sc, L.dinv, d_X, L.R, L.Z, L.P, L.AP,
                                                      L.done, L.part);
    QD_CHECK_LAUNCH();
    pcg_scalar_kernel<<<1, kScalarThreads, 0, s>>>(c, 2, L.part, L.sc, L.done, tol);
    QD_CHECK_LAUNCH();
    pcg_dir_kernel<<<c.blocks, c.threads, 0, s>>>(c, L.sc, L.Z, L.P, L.done);
    QD_CHECK_LAUNCH();
    if ((it + 1) % 16 == 0 || it + 1 == max_iter) {
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
