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
// Per iteration (S = [X W P], HS = [HX HW HP], MS = [MX MW MP]):
//   spmm_xp: explicit HX, MX, HP, MP (FP64 accumulation), residual
//            W = HX - MX Theta and its per-column norms
//   precond: W = T W (DST preconditioner, when the dot has a lattice)
//   ortho  : W = W - X (MX)^T W (M-orthogonal to X)
//   spmm   : HW = H W, MW = M W
//   gram   : per chunk, A_c = S^T HS and B_c = S^T MS (3B x 3B)
//   rr     : per dot (one CTA): convergence test, A = sum_c A_c, B = sum_c B_c,
//            orthonormal basis (Cholesky dropping dependent P directions, or
//            SVQB), the B lowest Ritz pairs (tridiagonalisation, bisection,
//            inverse iteration), Ritz coefficients Y -- all FP64 in shared
//            memory
//   update : X = S Y, P = [W P] Y_wp
// Recomputing the products of X and P every iteration (instead of updating
// them with the Ritz coefficients) keeps the residual consistent with X even
// when the basis is nearly dependent and the coefficients are large.
//
// Precision: QD_PREC_FP64 stores vectors in FP64.  QD_PREC_MIXED runs the
// iteration with FP32 vectors, FP32 (H, M) values and FP32 SpMM accumulation
// (Gram sums, Cholesky/SVQB and Rayleigh-Ritz in FP64) until the FP32 target
// or stagnation, then finishes with X, HX, MX in FP64 -- one FP64 product of
// X per iteration gives the residual and the Rayleigh-Ritz blocks of X, and X
// is updated in FP64 -- while the search directions W, P and their products
// stay FP32 (W's products by the FP32 SpMM).
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>
#include "common.h"
#include "spmm.cuh"
#include "dstprec.cuh"
#include "pipe.cuh"

namespace {

constexpr int kChunkRows = 1024;      // default rows per chunk (qd_lobpcg_opts.chunk_rows)

// Rows per chunk (the CTA unit of every row-parallel kernel): the option's
// value when it is a multiple of 64 in [256, 8192], else the default.
int chunk_rows_of(const qd_lobpcg_opts *opts) {
  const int c = opts ? opts->chunk_rows : 0;
  return (c >= 256 && c <= 8192 && c % 64 == 0) ? c : kChunkRows;
}
constexpr int kMaxB = 16;
constexpr int kMaxM = 3 * kMaxB;
constexpr int kStagWindow = 12;     // FP32 iterations without halving the estimate
constexpr double kTol32Floor = 1e-7; // FP32 phase target (estimated rel. eigenvalue error)
constexpr double kSafety = 1.0;
constexpr double kRelCap = 1e-2;
constexpr double kJacobiRel64 = 2e-15;   // relative Jacobi threshold, FP64 phase
constexpr double kJacobiRel32 = 1e-10;   // FP32 phase
constexpr double kJacobiRelMx = 1e-12;   // the mixed form's finishing phase
constexpr double kCholPivot32 = 1e-5;    // smallest Cholesky pivot of the scaled Gram (FP32 phase)
// ... in the mixed form's finishing phase: a basis of condition number below
// ~1e4 orthonormalised by Cholesky keeps its orthogonality to ~1e-12, well
// inside the 1e-9 eigenvalue target; worse bases go to SVQB
constexpr double kCholPivotMx = 1e-4;
#ifndef QD_SVQB_TAU64
#define QD_SVQB_TAU64 1e-12
#endif
#ifndef QD_SVQB_TAU32
#define QD_SVQB_TAU32 1e-6
#endif

struct Chunk {
  int dot, begin, end;
  int jacobi;       // the dot has no lattice: diagonal (Jacobi) preconditioning
};

struct DotState {
  int active;       // still iterating (either precision)
  int has_p;        // P block is populated
  int iters;        // total iterations (all phases)
  int iters_phase;  // iterations in the current phase
  int iters32;      // iterations spent in the FP32 phase
  int status;       // 0 running, 1 converged, 2 breakdown, 3 iteration cap
  int stag;         // iterations without 20% improvement (FP32 phase)
  int have_res;     // residual norms of the current X are available
  int chunk0, chunk1;
  double best;      // best max relative residual in this phase
  int launches[2][3];   // [FP32, FP64 phase][spmm, gram, update] launches that did work
  int run[2];       // iterating in the FP32 / FP64 phase (kernels of that precision work)
  int phase;        // 0 FP32, 1 FP64
  int switching;    // left the FP32 phase this iteration; X still to be converted
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
                            TV *W, TV *P, TV *HW, TV *MW, TV *HP, TV *MP, const double *X0,
                            int k) {
  const Chunk ch = chunks[blockIdx.x];
  const int r0 = row_off[ch.dot];
  for (int idx = threadIdx.x; idx < (ch.end - ch.begin) * B; idx += blockDim.x) {
    const int r = ch.begin + idx / B, j = idx % B;
    const uint64_t h = splitmix64(seed * 0x100000001b3ull + uint64_t(r - r0) * B + j);
    const double u = double(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    const size_t o = size_t(r) * B + j;
    // warm start: the caller's k vectors (row-major rows x k), random guard columns
    X[o] = (X0 && j < k) ? TV(X0[size_t(r) * k + j]) : TV(u);
    W[o] = P[o] = HW[o] = MW[o] = HP[o] = MP[o] = TV(0);
  }
}

// Row sums of the (scaled) FP32 H values, accumulated in FP64: the FP32
// SpMM differences H against each row's own entry and adds this sum back.
__global__ void rowsum32_kernel(int64_t n, const int32_t *__restrict__ rowptr,
                                const float2 *__restrict__ hm, float *__restrict__ rs) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    double a = 0.0;
    for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) a += double(hm[p].x);
    rs[r] = float(a);
  }
}

// Largest binary exponents of |H| and |M| (ilogb; zeros do not count).
__global__ void hm_exponent_kernel(int32_t nnz, const double *__restrict__ H,
                                   const double *__restrict__ M, int *e2) {
  int eh = INT_MIN, em = INT_MIN;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x) {
    const double h = H[p], m = M[p];
    if (h != 0.0) eh = max(eh, ilogb(h));
    if (m != 0.0) em = max(em, ilogb(m));
  }
  for (int o = 16; o > 0; o >>= 1) {
    eh = max(eh, __shfl_xor_sync(0xffffffffu, eh, o));
    em = max(em, __shfl_xor_sync(0xffffffffu, em, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&e2[0], eh);
    atomicMax(&e2[1], em);
  }
}

// The binary exponents of the FP32 pairs' scales (INT_MIN, from an all-zero
// matrix, counts as 0).
__device__ inline int hm_scale_exp(const int *e2, int i) {
  const int e = e2[i];
  return e == INT_MIN ? 0 : e;
}

// e2 = {INT_MIN, INT_MIN} before hm_exponent_kernel's maxima.
__global__ void hm_exponent_init_kernel(int *e2) {
  if (threadIdx.x < 2) e2[threadIdx.x] = INT_MIN;
}

// FP32 (H 2^-eh, M 2^-em) pairs of the FP32 phase's SpMMs, with the exponents
// read from the device (the host never waits for them).
__global__ void pack_hm32_kernel(int32_t nnz, const double *__restrict__ H,
                                 const double *__restrict__ M, const int *__restrict__ e2,
                                 float2 *__restrict__ hm) {
  const int eh = hm_scale_exp(e2, 0), em = hm_scale_exp(e2, 1);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += gridDim.x * blockDim.x)
    hm[p] = make_float2(float(scalbn(H[p], -eh)), float(scalbn(M[p], -em)));
}

template <typename TV, int B, typename MAT>
__global__ void __launch_bounds__(64 * (B / 4), 6)
spmm_chunk_kernel(const Chunk *chunks, const DotState *st, const int32_t *__restrict__ rowptr,
                  const int32_t *__restrict__ col, const MAT A, const TV *__restrict__ X,
                  TV *__restrict__ HX, TV *__restrict__ MX) {
  constexpr int G = B / 4;
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].run[sizeof(TV) == 8]) return;
  if (threadIdx.x == 0 && blockIdx.x == st[ch.dot].chunk0)
    const_cast<DotState *>(st)[ch.dot].launches[sizeof(TV) == 8][0]++;
  const int sub = threadIdx.x / G, g = threadIdx.x % G;
  const int rpp = blockDim.x / G;
  for (int r = ch.begin + sub; r < ch.end; r += rpp)
    qd::spmm_row<TV, B>(r, g, rowptr, col, A, X, HX, MX);
}

// Explicit products of the current X and P (no drift from implicit updates):
// HX, MX, HP, MP, the residual W = HX - MX Theta and per-chunk column norms
// sum r^2 and sum (Mx)^2.  2G threads per row: g < G own X columns, the rest P.
// TX is the storage of X and its products, TP that of the search directions
// P, HP, MP and of W: (double, double) in the plain FP64 form; (double, float)
// in the mixed form's finishing phase, where X and its products (the residual
// and the Rayleigh-Ritz blocks of X) stay FP64 and the search directions FP32.
// Accumulation is FP64 throughout.
template <typename TX, typename TP, int B, typename MAT>
__global__ void __launch_bounds__(128 * (B / 4), sizeof(TX) == 4 ? 3 : 2)
spmm_xp_kernel(const Chunk *chunks, const DotState *st, const int32_t *__restrict__ rowptr,
               const int32_t *__restrict__ col, const MAT A, const double *__restrict__ theta,
               const TX *__restrict__ X, const TP *__restrict__ P, TX *__restrict__ HX,
               TX *__restrict__ MX, TP *__restrict__ HP, TP *__restrict__ MP,
               TP *__restrict__ W, double *__restrict__ norms) {
  constexpr int G = B / 4;
  constexpr int G2 = 2 * G;
  constexpr int RPP = 64;   // rows per pass (blockDim = 64 * G2)
  constexpr int PH = sizeof(TX) == 8 ? 1 : 0;
  __shared__ double s_th[B];
  __shared__ double s_red[RPP * G2 * 8];
  const Chunk ch = chunks[blockIdx.x];
  const DotState &sd = st[ch.dot];
  if (!sd.run[PH]) return;
  const bool with_p = sd.has_p != 0;
  if (threadIdx.x == 0 && blockIdx.x == sd.chunk0)
    const_cast<DotState *>(st)[ch.dot].launches[PH][0]++;
  if (threadIdx.x < B) s_th[threadIdx.x] = theta[size_t(ch.dot) * B + threadIdx.x];
  __syncthreads();
  const int sub = threadIdx.x / G2, gg = threadIdx.x % G2;
  const bool isx = gg < G;
  const int g = isx ? gg : gg - G;
  // FP64 sums of squares (problems posed in SI units have squared residuals
  // far below FP32's range), kept in this thread's own shared-memory slots
  // slot layout [8][threads]: consecutive threads hit consecutive banks
  constexpr int NTX = RPP * G2;
  double *my_red = s_red + threadIdx.x;
#pragma unroll
  for (int c = 0; c < 8; ++c) my_red[c * NTX] = 0.0;
  // rows in sub-tiles of RPP, each taken in two halves of one parity (even
  // offsets, then odd): on the row-major lattice of a P2 mesh rows two apart
  // share their stencil, so the rows of one warp have the same number of
  // nonzeros and neighbouring columns
  const int ofs = sub < RPP / 2 ? 2 * sub : 2 * (sub - RPP / 2) + 1;
  for (int r = ch.begin + ofs; r < ch.end; r += RPP) {
    if (!isx && !with_p) {
      double z[4] = {0, 0, 0, 0};
      qd::V4<TP>::store(HP + size_t(r) * B + 4 * g, z);
      qd::V4<TP>::store(MP + size_t(r) * B + 4 * g, z);
      continue;
    }
    double h[4] = {0, 0, 0, 0}, m[4] = {0, 0, 0, 0};
    const int p0 = __ldg(rowptr + r), p1 = __ldg(rowptr + r + 1);
#pragma unroll 4
    for (int p = p0; p < p1; ++p) {
      const int j = __ldg(col + p);
      double hv, mv;
      A.get(p, hv, mv);
      double x[4];
      if (isx) qd::V4<TX>::load(X + size_t(j) * B + 4 * g, x);
      else qd::V4<TP>::load(P + size_t(j) * B + 4 * g, x);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        h[c] = fma(hv, x[c], h[c]);
        m[c] = fma(mv, x[c], m[c]);
      }
    }
    const size_t o = size_t(r) * B + 4 * g;
    if (isx) {
      double res[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        // residual from the stored (rounded) products, as the iteration sees them
        const double hq = double(TX(h[c])), mq = double(TX(m[c]));
        res[c] = hq - s_th[4 * g + c] * mq;
        my_red[(2 * c) * NTX] += res[c] * res[c];
        my_red[(2 * c + 1) * NTX] += mq * mq;
      }
      qd::V4<TX>::store(HX + o, h);
      qd::V4<TX>::store(MX + o, m);
      qd::V4<TP>::store(W + o, res);
    } else {
      qd::V4<TP>::store(HP + o, h);
      qd::V4<TP>::store(MP + o, m);
    }
  }
  // per-chunk column norms (fixed-order reduction over the CTA's rows)
  __syncthreads();
  if (threadIdx.x < B) {
    const int j = threadIdx.x, gj = j / 4, cj = j % 4;
    double a = 0.0, b = 0.0;
    for (int sr = 0; sr < RPP; ++sr) {
      const int t = sr * G2 + gj;
      a += s_red[(2 * cj) * NTX + t];
      b += s_red[(2 * cj + 1) * NTX + t];
    }
    norms[size_t(blockIdx.x) * 2 * B + j] = a;
    norms[size_t(blockIdx.x) * 2 * B + B + j] = b;
  }
}

// ---------------------------------------------------------------------------
// FP32-phase SpMM with every operand of a sub-tile staged in shared memory.
// A sub-tile of rows [a, b) needs the nonzeros [rowptr[a], rowptr[b]) and the
// vector rows its columns name.  On a lattice those rows form a few runs (one
// per lattice line of the stencil: five for a P2 sub-tile of 64 rows inside
// one line, about 260 rows in all), so a plan built once per solve
// (stage_plan_kernel) lists each sub-tile's runs of rows and rewrites every
// column index as a position in the staged copy (16-bit).  The kernel then
// fetches, per sub-tile, the positions, the FP32 (H, M) pairs and the runs of
// X (and P) by 1-D bulk copies into a 2-stage mbarrier pipeline, and every
// gather of the nonzero loop is a shared-memory load.  A sub-tile with more
// nonzeros, runs or rows than a stage holds reads everything from global
// memory instead (same arithmetic, same results).
// XP: products of X and P with the residual W = HX - MX Theta and per-chunk
// norms, in sub-tiles of 64 rows (six threads per row); otherwise the
// products of one block (W -> HW, MW) in sub-tiles of 128 rows (three threads
// per row).  Either way a CTA has 32 B threads and two fit on an SM (B <= 12).
// ---------------------------------------------------------------------------
constexpr int kMaxSeg = 6;                  // runs of rows per sub-tile
constexpr int kCsrStages = 2;
constexpr int kPlanSlots = 4;               // staged plan records (ring)

// The staging plan of one sub-tile: nseg < 0 if it is read from global
// memory; else its nonzeros [q0, q1) and runs [lo[s], lo[s] + len[s]) of
// vector rows, stored one after another (total rows).
struct SubPlan {
  int nseg, total, q0, q1;
  int lo[kMaxSeg];
  int len[kMaxSeg];
};
static_assert(sizeof(SubPlan) == 64, "one 64-byte record per sub-tile");

// Sub-tiles of SUBR rows: staged nonzeros and vector rows per sub-tile (on a
// P2 lattice at most 896 / 342 for 64 rows and 1792 / 649 for 128).
template <int SUBR> struct StageCap;
template <> struct StageCap<64> {
  static constexpr int NNZ = 1024, ROWS = 384;
};
template <> struct StageCap<128> {
  static constexpr int NNZ = 2048, ROWS = 672;
};

template <int B, int NBLK, int SUBR> struct SpmmStage {
  static constexpr int CAP = StageCap<SUBR>::NNZ;
  static constexpr int ROWS = StageCap<SUBR>::ROWS;
  static constexpr int POS = CAP + 16;            // uint16 slots (16-byte rounding slack)
  static constexpr int HM = CAP + 4;              // float2 slots
  // Consecutive staged blocks are 12 floats further apart than their size:
  // with B = 12, rows j of X and P then fall on disjoint banks, so the
  // warp-wide gathers (three threads per row and block) are conflict-free.
  static constexpr int SKEW = 12;
  static constexpr size_t POS_OFF = 0;
  static constexpr size_t HM_OFF = size_t(POS) * 2;
  static constexpr size_t ROW_OFF = HM_OFF + size_t(HM) * 8;
  static constexpr size_t BLK = size_t(ROWS * B + SKEW) * 4;
  static constexpr size_t STAGE = ROW_OFF + NBLK * BLK;
  static constexpr size_t META_OFF = kCsrStages * STAGE;
  // barriers, then per stage: position base, pair base, staged flag, and
  // the offset from a row of the sub-tile itself to its staged position
  static constexpr size_t BYTES = META_OFF + kCsrStages * 8 + kCsrStages * 4 * 4;
  static_assert(HM_OFF % 16 == 0 && ROW_OFF % 16 == 0 && BLK % 16 == 0 && STAGE % 16 == 0,
                "bulk-copy destinations must be 16-byte aligned");
};

// One warp per sub-tile of SUBR rows (chunk c, sub-tile i at record
// c * spc + i): the runs
// of the column indices of its nonzeros and their staged positions.  Runs are
// found as maximal runs of touched 8-row blocks (so gaps of fewer than 8
// untouched rows are staged with them), then trimmed to the smallest and
// largest column they hold.
template <int SUBR>
__global__ void __launch_bounds__(256)
stage_plan_kernel(const Chunk *chunks, int nchunks, int spc, const int32_t *__restrict__ rowptr,
                  const int32_t *__restrict__ col, SubPlan *__restrict__ plan,
                  uint16_t *__restrict__ pos16) {
  constexpr int NW = 64;   // bitmap words per warp: 2048 blocks of 8 rows
  __shared__ uint32_t s_bits[8][NW];
  __shared__ int s_start[8][kMaxSeg];
  __shared__ int s_lo[8][kMaxSeg], s_hi[8][kMaxSeg], s_off[8][kMaxSeg];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t = int64_t(blockIdx.x) * 8 + w;
  if (t >= int64_t(nchunks) * spc) return;   // whole warps; only warp syncs below
  const Chunk ch = chunks[t / spc];
  const int a = ch.begin + int(t % spc) * SUBR;
  SubPlan *out = plan + t;
  if (a >= ch.end) {
    if (lane == 0) out->nseg = -1;
    return;
  }
  const int b = min(a + SUBR, ch.end);
  const int q0 = __ldg(rowptr + a), q1 = __ldg(rowptr + b);
  int cmin = INT_MAX, cmax = INT_MIN;
  for (int p = q0 + lane; p < q1; p += 32) {
    const int j = __ldg(col + p);
    cmin = min(cmin, j);
    cmax = max(cmax, j);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
    cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  }
  bool ok = q1 > q0 && q1 - q0 <= StageCap<SUBR>::NNZ &&
            int64_t(cmax) - cmin < int64_t(NW) * 32 * 8;
  if (ok) {
    for (int k = lane; k < NW; k += 32) s_bits[w][k] = 0u;
    __syncwarp();
    for (int p = q0 + lane; p < q1; p += 32) {
      const int blk = (__ldg(col + p) - cmin) >> 3;
      atomicOr(&s_bits[w][blk >> 5], 1u << (blk & 31));
    }
    __syncwarp();
    // lane l holds blocks [64 l, 64 l + 64); a run starts at a touched block
    // whose predecessor is untouched
    const uint64_t v = uint64_t(s_bits[w][2 * lane]) | (uint64_t(s_bits[w][2 * lane + 1]) << 32);
    const uint64_t prev_top = __shfl_up_sync(0xffffffffu, v >> 63, 1);
    const uint64_t starts = v & ~((v << 1) | (lane > 0 ? prev_top : 0ull));
    const int cnt = __popcll(starts);
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int nseg = __shfl_sync(0xffffffffu, incl, 31);
    ok = nseg <= kMaxSeg;
    if (ok) {
      int e = incl - cnt;
      for (uint64_t s = starts; s; s &= s - 1) s_start[w][e++] = 64 * lane + __ffsll(s) - 1;
      if (lane < nseg) {
        s_lo[w][lane] = INT_MAX;
        s_hi[w][lane] = INT_MIN;
      }
      __syncwarp();
      for (int p = q0 + lane; p < q1; p += 32) {
        const int j = __ldg(col + p), blk = (j - cmin) >> 3;
        int sg = 0;
        while (sg + 1 < nseg && s_start[w][sg + 1] <= blk) ++sg;
        atomicMin(&s_lo[w][sg], j);
        atomicMax(&s_hi[w][sg], j);
      }
      __syncwarp();
      int total = 0;
      int own = 0;   // the sub-tile's own rows lie in one run (their diagonal entries)
      if (lane == 0) {
        for (int sg = 0; sg < nseg; ++sg) {
          s_off[w][sg] = total;
          total += s_hi[w][sg] - s_lo[w][sg] + 1;
          own |= s_lo[w][sg] <= a && b - 1 <= s_hi[w][sg];
        }
      }
      total = __shfl_sync(0xffffffffu, total, 0);
      own = __shfl_sync(0xffffffffu, own, 0);
      __syncwarp();
      ok = total <= StageCap<SUBR>::ROWS && own;
      if (ok) {
        for (int p = q0 + lane; p < q1; p += 32) {
          const int j = __ldg(col + p), blk = (j - cmin) >> 3;
          int sg = 0;
          while (sg + 1 < nseg && s_start[w][sg + 1] <= blk) ++sg;
          pos16[p] = uint16_t(s_off[w][sg] + j - s_lo[w][sg]);
        }
        if (lane < nseg) {
          out->lo[lane] = s_lo[w][lane];
          out->len[lane] = s_hi[w][lane] - s_lo[w][lane] + 1;
        }
        if (lane == 0) {
          out->nseg = nseg;
          out->total = total;
          out->q0 = q0;
          out->q1 = q1;
        }
      }
    }
  }
  if (!ok && lane == 0) out->nseg = -1;
}

template <int B, bool XP>
__global__ void __launch_bounds__(32 * B, B <= 12 ? 2 : 1)
spmm32s_kernel(const Chunk *chunks, const DotState *st, const int32_t *__restrict__ rowptr,
               const int32_t *__restrict__ col32, const uint16_t *__restrict__ pos16,
               const SubPlan *__restrict__ plan, int spc, const float2 *__restrict__ hm32,
               const float *__restrict__ rs32, const int *__restrict__ hm_e,
               const double *__restrict__ theta, const float *__restrict__ X,
               const float *__restrict__ P, float *__restrict__ HX, float *__restrict__ MX,
               float *__restrict__ HP, float *__restrict__ MP, float *__restrict__ W,
               double *__restrict__ norms, int *wait_err, int ph) {
  constexpr int G = B / 4;
  constexpr int G2 = XP ? 2 * G : G;
  constexpr int SUBR = XP ? 64 : 128;   // rows per sub-tile: 32 B threads either way
  constexpr int NT = SUBR * G2;
  constexpr int NBLK = XP ? 2 : 1;
  using SS = SpmmStage<B, NBLK, SUBR>;
  static_assert(!XP || size_t(NT) * 8 * sizeof(double) <= SS::META_OFF,
                "the norm slots reuse the stage buffers");
  extern __shared__ __align__(128) unsigned char dsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(dsm + SS::META_OFF);
  int *s_pbase = reinterpret_cast<int *>(full + kCsrStages);
  int *s_hbase = s_pbase + kCsrStages;
  int *s_staged = s_hbase + kCsrStages;
  int *s_obase = s_staged + kCsrStages;
  __shared__ double s_th[B];
  __shared__ __align__(16) SubPlan s_plan[kPlanSlots];

  // ph: the phase whose dots this launch serves (the products of X and P only
  // in the FP32 phase; W's products also in the mixed form's finishing phase)
  const Chunk ch = chunks[blockIdx.x];
  const DotState &sd = st[ch.dot];
  if (!sd.run[ph]) return;
  const bool with_p = sd.has_p != 0;
  const int tid = threadIdx.x;
  if (tid == 0 && blockIdx.x == sd.chunk0)
    const_cast<DotState *>(st)[ch.dot].launches[ph][0]++;
  if (XP && tid < B) s_th[tid] = theta[size_t(ch.dot) * B + tid];
  const int sub = tid / G2, gg = tid % G2;
  const bool isx = gg < G;
  const int g = isx ? gg : gg - G;
  // scales 2^e of the FP32 (H, M) pairs
  const float fsh = ldexpf(1.f, hm_scale_exp(hm_e, 0)), fsm = ldexpf(1.f, hm_scale_exp(hm_e, 1));
  // FP64 sums of squares of this thread's rows (problems posed in SI units
  // have squared residuals far below FP32's range): r^2, (Mx)^2 per column
  double red[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) red[c] = 0.0;
  const int nsub = (ch.end - ch.begin + SUBR - 1) / SUBR;
  if (tid == 0) {
    for (int i = 0; i < kCsrStages; ++i) qd::tc::mbar_init(&full[i], 1);
    qd::tc::fence_mbar_init();
  }
  __syncthreads();
  const int nblk = (XP && with_p) ? 2 : 1;   // blocks staged (P only once populated)
  // Thread 0 issues sub-tile i's copies from its plan record pl; each stage
  // also brings in the record of the sub-tile issued after it (i + stages),
  // so that no global load stands between a sub-tile's barrier and the next
  // issue.
  const SubPlan *plan_c = plan + size_t(blockIdx.x) * spc;
  auto issue = [&](int i, const SubPlan &pl) {   // thread 0
    const int sst = i % kCsrStages;
    unsigned char *sb = dsm + size_t(sst) * SS::STAGE;
    const int nseg = pl.nseg;
    const bool next = i + kCsrStages < nsub;
    const uint32_t pr = next ? uint32_t(sizeof(SubPlan)) : 0u;
    if (nseg >= 0) {
      const int a = ch.begin + i * SUBR;
      const int q0 = pl.q0, q1 = pl.q1;
      const int pb = q0 & ~7, pe = (q1 + 7) & ~7;
      const int hb = q0 & ~1, he = (q1 + 1) & ~1;
      s_pbase[sst] = pb;
      s_hbase[sst] = hb;
      s_staged[sst] = 1;
      const uint32_t pbytes = uint32_t(pe - pb) * 2u, hbytes = uint32_t(he - hb) * 8u;
      const uint32_t rbytes = uint32_t(pl.total) * B * 4u;
      int off = 0, obase = 0;
      for (int sg = 0; sg < nseg; ++sg) {   // the run of the sub-tile's own rows
        const int lo = pl.lo[sg], len = pl.len[sg];
        if (a >= lo && a < lo + len) obase = off - lo;
        off += len;
      }
      s_obase[sst] = obase;
      qd::tc::mbar_arrive_expect_tx(&full[sst], pbytes + hbytes + nblk * rbytes + pr);
      qd::tc::bulk_g2s(sb + SS::POS_OFF, pos16 + pb, pbytes, &full[sst]);
      qd::tc::bulk_g2s(sb + SS::HM_OFF, hm32 + hb, hbytes, &full[sst]);
      off = 0;
      for (int sg = 0; sg < nseg; ++sg) {
        const int lo = pl.lo[sg], len = pl.len[sg];
        for (int k = 0; k < nblk; ++k)
          qd::tc::bulk_g2s(sb + SS::ROW_OFF + k * SS::BLK + size_t(off) * B * 4,
                           (k ? P : X) + size_t(lo) * B, uint32_t(len) * B * 4u, &full[sst]);
        off += len;
      }
    } else {
      s_staged[sst] = 0;
      qd::tc::mbar_arrive_expect_tx(&full[sst], pr);
    }
    if (next)
      qd::tc::bulk_g2s(&s_plan[(i + kCsrStages) % kPlanSlots], plan_c + i + kCsrStages,
                       uint32_t(sizeof(SubPlan)), &full[sst]);
  };
  if (tid == 0)
    for (int i = 0; i < kCsrStages && i < nsub; ++i) issue(i, plan_c[i]);
  bool ok = true;
  for (int i = 0; i < nsub; ++i) {
    const int sst = i % kCsrStages;
    // the sub-tile's rows in two halves of one parity each (even offsets,
    // then odd): on the row-major lattice of a P2 mesh, rows two apart have
    // the same stencil, so the k-th neighbours gathered by one warp lie close
    const int ofs = sub < SUBR / 2 ? 2 * sub : 2 * (sub - SUBR / 2) + 1;
    const int r = ch.begin + i * SUBR + ofs;
    const bool live = r < ch.end;
    int p0 = 0, p1 = 0;
    float rs = 0.f;
    if (live) {
      p0 = __ldg(rowptr + r);
      p1 = __ldg(rowptr + r + 1);
      rs = __ldg(rs32 + r);
    }
    ok = qd::tc::mbar_wait(&full[sst], (i / kCsrStages) & 1, qd::kPipeWaitNs) && ok;
    if (ok && live) {
      if (XP && !isx && !with_p) {
        const double z[4] = {0, 0, 0, 0};
        qd::V4<float>::store(HP + size_t(r) * B + 4 * g, z);
        qd::V4<float>::store(MP + size_t(r) * B + 4 * g, z);
      } else {
        const int blk = (XP && !isx) ? 1 : 0;
        const float *src = blk ? P : X;
        const bool staged = s_staged[sst] != 0;
        const unsigned char *sb = dsm + size_t(sst) * SS::STAGE;
        const float *rows =
            reinterpret_cast<const float *>(sb + SS::ROW_OFF + blk * SS::BLK) + 4 * g;
        // FP32 arithmetic, H differenced against the row's own entry:
        //   (H x)_i = sum_j H_ij (x_j - x_i) + (sum_j H_ij) x_i
        // The stiffness part of H has (near) zero row sums, so the terms are
        // small where x is smooth and FP32 accumulation stays ~1e-6 accurate
        // relative to H x (undifferenced, the terms exceed H x by up to 1e4).
        const float4 xi =
            staged ? *reinterpret_cast<const float4 *>(rows + (r + s_obase[sst]) * B)
                   : __ldg(reinterpret_cast<const float4 *>(src + size_t(r) * B + 4 * g));
        float h[4] = {0.f, 0.f, 0.f, 0.f}, m[4] = {0.f, 0.f, 0.f, 0.f};
        auto row = [&](auto getx, auto getv) {
#pragma unroll 4
          for (int p = p0; p < p1; ++p) {
            const float2 v = getv(p);
            const float4 xj = getx(p);
            h[0] = fmaf(v.x, xj.x - xi.x, h[0]);
            h[1] = fmaf(v.x, xj.y - xi.y, h[1]);
            h[2] = fmaf(v.x, xj.z - xi.z, h[2]);
            h[3] = fmaf(v.x, xj.w - xi.w, h[3]);
            m[0] = fmaf(v.y, xj.x, m[0]);
            m[1] = fmaf(v.y, xj.y, m[1]);
            m[2] = fmaf(v.y, xj.z, m[2]);
            m[3] = fmaf(v.y, xj.w, m[3]);
          }
        };
        if (staged) {
          const uint16_t *ps = reinterpret_cast<const uint16_t *>(sb + SS::POS_OFF) - s_pbase[sst];
          const float2 *hs = reinterpret_cast<const float2 *>(sb + SS::HM_OFF) - s_hbase[sst];
          row([&](int p) { return *reinterpret_cast<const float4 *>(rows + int(ps[p]) * B); },
              [&](int p) { return hs[p]; });
        } else {
          row([&](int p) {
                return __ldg(reinterpret_cast<const float4 *>(src + size_t(__ldg(col32 + p)) * B +
                                                              4 * g));
              },
              [&](int p) { return __ldg(hm32 + p); });
        }
        h[0] = fmaf(rs, xi.x, h[0]);
        h[1] = fmaf(rs, xi.y, h[1]);
        h[2] = fmaf(rs, xi.z, h[2]);
        h[3] = fmaf(rs, xi.w, h[3]);
        const size_t o = size_t(r) * B + 4 * g;
        // back to the matrices' own scale (powers of two: exact)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          h[c] *= fsh;
          m[c] *= fsm;
        }
        if (XP && isx) {
          double res[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            // residual from the stored (rounded) products, as the iteration sees them
            const double hq = double(h[c]), mq = double(m[c]);
            res[c] = hq - s_th[4 * g + c] * mq;
            red[2 * c] += res[c] * res[c];
            red[2 * c + 1] += mq * mq;
          }
          *reinterpret_cast<float4 *>(HX + o) = make_float4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<float4 *>(MX + o) = make_float4(m[0], m[1], m[2], m[3]);
          qd::V4<float>::store(W + o, res);
        } else {
          float *oh = XP ? HP : HX, *om = XP ? MP : MX;
          *reinterpret_cast<float4 *>(oh + o) = make_float4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<float4 *>(om + o) = make_float4(m[0], m[1], m[2], m[3]);
        }
      }
    }
    __syncthreads();   // stage sst consumed
    if (tid == 0 && ok && i + kCsrStages < nsub)
      issue(i + kCsrStages, s_plan[(i + kCsrStages) % kPlanSlots]);
  }
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicOr(wait_err, 1);
      for (int i = max(0, nsub - kCsrStages); i < nsub; ++i)
        qd::tc::mbar_wait(&full[i % kCsrStages], (i / kCsrStages) & 1, qd::kPipeWaitNs);
    }
    return;
  }
  if (XP) {
    // per-chunk column norms (fixed-order reduction over the CTA's rows); the
    // slots [8][threads] take the stage buffers, whose copies have all landed
    double *s_red = reinterpret_cast<double *>(dsm);
#pragma unroll
    for (int c = 0; c < 8; ++c) s_red[c * NT + tid] = red[c];
    __syncthreads();
    if (tid < B) {
      const int j = tid, gj = j / 4, cj = j % 4;
      double a = 0.0, b = 0.0;
      for (int sr = 0; sr < SUBR; ++sr) {
        const int t = sr * G2 + gj;
        a += s_red[(2 * cj) * NT + t];
        b += s_red[(2 * cj + 1) * NT + t];
      }
      norms[size_t(blockIdx.x) * 2 * B + j] = a;
      norms[size_t(blockIdx.x) * 2 * B + B + j] = b;
    }
  }
}

// ---------------------------------------------------------------------------
// Gram partials: per chunk A_c = S^T HS, B_c = S^T MS  (m = 3B, full m x m)
// ---------------------------------------------------------------------------

// Opt a kernel into `bytes` of dynamic shared memory (once per kernel).
template <auto Kern>
cudaError_t smem_attr(size_t bytes) {
  static std::once_flag once;
  static cudaError_t e = cudaSuccess;
  std::call_once(once, [bytes] {
    e = cudaFuncSetAttribute(Kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  });
  return e;
}

// Gram tasks: one upper-triangle 4x4 block (bi <= bj) of S^T HS or of S^T MS
// per thread (NT2 = 2 NT tasks), RG row groups.  One matrix per thread keeps
// the FP64 accumulators at 16 values, so two CTAs fit on an SM.
template <typename TV, int B> struct GramCfg {
  static constexpr int m = 3 * B;
  static constexpr int NB = m / 4;
  static constexpr int NT = NB * (NB + 1) / 2;            // upper-triangle 4x4 blocks
  static constexpr int NT2 = 2 * NT;                      // of S^T HS, then of S^T MS
  static constexpr int TARGET = sizeof(TV) == 8 ? 256 : 384;
  static constexpr int RG = (TARGET / NT2) > 0 ? (TARGET / NT2) : 1;
  static constexpr int THREADS = ((NT2 * RG + 31) / 32) * 32;
};

// The Gram kernel streams the 9 vector blocks X W P HX HW HP MX MW MP of each
// sub-tile through a 3-stage bulk-copy pipeline.
// Four consecutive elements of a staged row in shared memory, as one 16-byte
// (FP32) or two 16-byte (FP64) loads.  Stage tiles start 16-byte aligned, row
// pitches are B elements (B % 4 == 0) and column groups start at multiples of
// 4 elements, so every such group is 16-byte aligned.
template <typename TV> __device__ inline void lds4(const TV *p, TV (&v)[4]);
template <> __device__ inline void lds4<float>(const float *p, float (&v)[4]) {
  const float4 a = *reinterpret_cast<const float4 *>(p);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}
template <> __device__ inline void lds4<double>(const double *p, double (&v)[4]) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0];
  const double2 b = reinterpret_cast<const double2 *>(p)[1];
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}

template <typename TV, int B> using GramPipe = qd::BlockPipe<TV, B, 9, (sizeof(TV) == 8 ? 32 : 64), 3>;

// Each thread owns one upper-triangle 4x4 block (bi <= bj) of both S^T HS and
// S^T MS for a slice (row group rg) of every sub-tile's rows, accumulating
// in TV within a sub-tile and in FP64 across sub-tiles.  Off-diagonal blocks
// are written to both (bi, bj) and (bj, bi), so the per-chunk partial holds
// the full symmetric matrices.
template <typename TV, int B>
__global__ void __launch_bounds__(GramCfg<TV, B>::THREADS, 2)
gram_kernel(const Chunk *chunks, const DotState *st, const TV *X, const TV *W, const TV *P,
            const TV *HX, const TV *HW, const TV *HP, const TV *MX, const TV *MW, const TV *MP,
            double *partial, int *wait_err) {
  using C = GramCfg<TV, B>;
  using PP = GramPipe<TV, B>;
  constexpr int m = C::m, NB = C::NB, NT = C::NT, NT2 = C::NT2, RG = C::RG;
  constexpr int BLK = PP::BLKP;   // block stride inside a stage
  extern __shared__ __align__(128) unsigned char dsm[];

  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].run[sizeof(TV) == 8]) return;
  const int tid = threadIdx.x;
  if (tid == 0 && blockIdx.x == st[ch.dot].chunk0)
    const_cast<DotState *>(st)[ch.dot].launches[sizeof(TV) == 8][1]++;
  const bool worker = tid < NT2 * RG;
  const int task2 = tid % NT2, rg = tid / NT2;
  const int which = task2 / NT, task = task2 % NT;   // which: 0 S^T HS, 1 S^T MS
  // task -> (bi, bj) with bi <= bj
  int bi = 0, rem = task;
  while (rem >= NB - bi) {
    rem -= NB - bi;
    ++bi;
  }
  const int bj = bi + rem;
  // element offsets of this thread's 4 columns inside a stage (B % 4 == 0,
  // so a group of 4 columns never straddles two blocks)
  const int offS = ((4 * bi) / B) * BLK + (4 * bi) % B;
  const int offR = (3 + 3 * which + (4 * bj) / B) * BLK + (4 * bj) % B;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;

  const TV *src[9] = {X, W, P, HX, HW, HP, MX, MW, MP};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (worker && ok) {
      const int nr = pipe.rows(i);
      const TV *sb = pipe.tile(i, 0);
      TV t[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) t[a][b] = TV(0);
      for (int row = rg; row < nr; row += RG) {
        TV sa[4], rb[4];
        lds4(sb + offS + row * B, sa);
        lds4(sb + offR + row * B, rb);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) t[a][b] = fma(sa[a], rb[b], t[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += double(t[a][b]);
    }
    pipe.release(i, ok);
  }
  if (!pipe.finish(ok, wait_err)) return;
  double *out = partial + size_t(blockIdx.x) * 2 * m * m;
  if (RG > 1) {
    double *red = reinterpret_cast<double *>(dsm);   // NT2 * 16 doubles < one stage
    for (int g = 1; g < RG; ++g) {
      if (worker && rg == g) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) red[task2 * 16 + a * 4 + b] = acc[a][b];
      }
      __syncthreads();
      if (worker && rg == 0) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] += red[task2 * 16 + a * 4 + b];
      }
      __syncthreads();
    }
  }
  if (worker && rg == 0) {
    double *o = out + size_t(which) * m * m;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int i = 4 * bi + a, j = 4 * bj + b;
        o[i * m + j] = acc[a][b];
        if (bi != bj) o[j * m + i] = acc[a][b];
      }
  }
}

// ---------------------------------------------------------------------------
// Rayleigh-Ritz per dot (FP64, one CTA of 256 threads, m <= 48)
// ---------------------------------------------------------------------------

struct RRParams {
  int k;
  double tol32;    // FP32-phase target (then the dot switches to FP64)
  double tol;      // relative residual tolerance for this phase
  int max_iter;    // total iteration cap per dot
  int stag_window; // FP32 iterations without halving the estimate before the switch
  double eig_scale; // floor of |theta| in the relative error estimate (0: none)
  int mixed;        // the mixed form: its finishing phase has FP32 W and P blocks
};

// Cyclic Jacobi eigensolver for a symmetric n x n matrix A (leading dimension
// ld, shared memory) with round-robin pairing; V (ld) receives the
// eigenvectors as columns, A's diagonal the eigenvalues.  A pair is rotated
// only while |a_pq| > rel sqrt(|a_pp a_qq|) (the relative threshold of
// Demmel and Veselic: with rel = 2e-15 tiny eigenvalues of a scaled SPD Gram
// matrix come out with high relative accuracy) and |a_pq| > 1e-18 ||A||_F
// (below that the entry is rounding noise and rotating it only costs
// sweeps); the sweeps stop when a sweep rotates nothing.
// One round = the ne/2 disjoint pairs of the schedule (odd n adds a dummy
// index that never rotates), in two phases separated by barriers:
//   (1) pair t computes its rotation R_t from the current a_pp, a_qq, a_pq;
//   (2) every 2x2 block (t, u), t <= u, becomes R_t^T A_tu R_u in one step
//       (it depends only on its own old entries and the two rotations; the
//       annihilated a_pq of a diagonal block is set to 0), mirrored to (u, t),
//       and V's columns p, q are rotated.
__device__ void jacobi_cta(double *A, double *V, int n, int ld, double rel, double *s_red,
                           double *s_c, double *s_s, int *s_p, int *s_q) {
  const int tid = threadIdx.x, nt = blockDim.x;
  // "some pair rotated" flag per sweep, double-buffered: sweep k sets slot
  // k & 1 and clears the other slot behind a barrier for sweep k + 1
  __shared__ int s_rot[2];
  if (tid == 0) s_rot[0] = s_rot[1] = 0;
  for (int idx = tid; idx < n * n; idx += nt) {
    const int i = idx / n, j = idx % n;
    V[i * ld + j] = (i == j) ? 1.0 : 0.0;
  }
  // absolute floor: off-diagonal entries below 1e-18 ||A||_F are rounding noise
  double fro = 0.0;
  for (int idx = tid; idx < n * n; idx += nt) {
    const double v = A[(idx / n) * ld + idx % n];
    fro += v * v;
  }
  s_red[tid] = fro;
  __syncthreads();
  for (int w = nt / 2; w > 0; w >>= 1) {
    if (tid < w) s_red[tid] += s_red[tid + w];
    __syncthreads();
  }
  const double floor_abs = 1e-18 * sqrt(s_red[0]);
  __syncthreads();
  const int ne = (n + 1) & ~1;   // even count including the dummy
  if (ne < 2) return;
  const int np = ne / 2;
  const int nblk = np * (np + 1) / 2;
  // this thread's 2x2 blocks (t <= u) and V tasks (pair t, row i): fixed for
  // all rounds, decoded once (nblk <= 300 and np * n <= 1152 for n <= 48)
  constexpr int kBT = 2, kVT = 5;
  int bt[kBT], bu[kBT], vt[kVT], vi[kVT];
#pragma unroll
  for (int q = 0; q < kBT; ++q) {
    const int b = tid + q * nt;
    bt[q] = -1;
    bu[q] = -1;
    if (b < nblk) {
      int t = 0, rem = b;
      while (rem >= np - t) {
        rem -= np - t;
        ++t;
      }
      bt[q] = t;
      bu[q] = t + rem;
    }
  }
#pragma unroll
  for (int q = 0; q < kVT; ++q) {
    const int idx = tid + q * nt;
    vt[q] = idx < np * n ? idx / n : -1;
    vi[q] = idx < np * n ? idx % n : 0;
  }
  for (int sweep = 0; sweep < 60; ++sweep) {
    const int cur = sweep & 1;
    for (int round = 0; round < ne - 1; ++round) {
      // (1) rotations of this round's pairs
      if (tid < np) {
        int p, q;
        if (tid == 0) {
          p = 0;
          q = 1 + (round % (ne - 1));
        } else {
          p = 1 + ((tid + round) % (ne - 1));
          q = 1 + ((ne - 1 - tid + round) % (ne - 1));
        }
        if (p > q) {
          const int t = p; p = q; q = t;
        }
        double c = 1.0, sn = 0.0;
        if (q < n) {
          const double apq = A[p * ld + q];
          const double app = A[p * ld + p], aqq = A[q * ld + q];
          if (fabs(apq) > floor_abs && fabs(apq) > rel * sqrt(fabs(app * aqq))) {
            const double tau = (aqq - app) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = rsqrt(1.0 + t * t);
            sn = t * c;
            s_rot[cur] = 1;
          }
        }
        s_c[tid] = c;
        s_s[tid] = sn;
        s_p[tid] = p;
        s_q[tid] = q;
      }
      __syncthreads();
      // (2) 2x2 blocks (t <= u) of A, then the columns of V
      if (round == 0 && tid == 0) s_rot[cur ^ 1] = 0;
#pragma unroll
      for (int qb = 0; qb < kBT; ++qb) {
        const int t = bt[qb], u = bu[qb];
        if (t < 0) continue;
        const int pt = s_p[t], qt = s_q[t], pu = s_p[u], qu = s_q[u];
        const double ct = s_c[t], st_ = s_s[t], cu = s_c[u], su = s_s[u];
        if (ct == 1.0 && st_ == 0.0 && cu == 1.0 && su == 0.0) continue;   // nothing rotates
        const bool qtv = qt < n, quv = qu < n;
        const double a00 = A[pt * ld + pu];
        const double a01 = quv ? A[pt * ld + qu] : 0.0;
        const double a10 = qtv ? A[qt * ld + pu] : 0.0;
        const double a11 = (qtv && quv) ? A[qt * ld + qu] : 0.0;
        // rows: [r0; r1] = R_t^T [a0x; a1x] with R = [[c, s], [-s, c]]
        const double r00 = ct * a00 - st_ * a10, r01 = ct * a01 - st_ * a11;
        const double r10 = st_ * a00 + ct * a10, r11 = st_ * a01 + ct * a11;
        // columns: [.. x0, .. x1] R_u
        double n00 = cu * r00 - su * r01, n01 = su * r00 + cu * r01;
        double n10 = cu * r10 - su * r11, n11 = su * r10 + cu * r11;
        if (t == u) {
          if (st_ != 0.0) n01 = n10 = 0.0;   // the annihilated entry
          A[pt * ld + pt] = n00;
          if (qtv) {
            A[qt * ld + qt] = n11;
            A[pt * ld + qt] = n01;
            A[qt * ld + pt] = n10;
          }
        } else {
          A[pt * ld + pu] = n00;
          A[pu * ld + pt] = n00;
          if (quv) {
            A[pt * ld + qu] = n01;
            A[qu * ld + pt] = n01;
          }
          if (qtv) {
            A[qt * ld + pu] = n10;
            A[pu * ld + qt] = n10;
          }
          if (qtv && quv) {
            A[qt * ld + qu] = n11;
            A[qu * ld + qt] = n11;
          }
        }
      }
#pragma unroll
      for (int qv = 0; qv < kVT; ++qv) {
        const int t = vt[qv], i = vi[qv];
        if (t < 0) continue;
        const int p = s_p[t], q = s_q[t];
        const double c = s_c[t], sn = s_s[t];
        if (q >= n || sn == 0.0) continue;
        const double va = V[i * ld + p], vb = V[i * ld + q];
        V[i * ld + p] = c * va - sn * vb;
        V[i * ld + q] = sn * va + c * vb;
      }
      __syncthreads();
    }
    if (!s_rot[cur]) break;
  }
  __syncthreads();
}

// The nsel lowest eigenpairs of the symmetric n x n matrix A (shared memory,
// leading dimension ld; destroyed), by
//   (1) Householder reduction to tridiagonal form T = H^T A H, the reflector
//       vectors kept in A's columns below the subdiagonal (3 barriers per
//       column; 8 lanes per row for the matrix-vector product, the rank-2
//       update's scalar reduced by every warp for itself);
//   (2) bisection on Sturm counts of T for all nsel eigenvalues at once, a
//       group of L = min(32, blockDim / nsel) threads per eigenvalue testing
//       L points of its interval per round ((L+1)-way multisection);
//   (3) inverse iteration on T - lambda_j I (Gaussian elimination with row
//       interchanges, two steps from a fixed pseudo-random start), one
//       thread per eigenvalue, then classical Gram-Schmidt applied twice
//       over the nsel vectors in ascending order (orthonormal also inside
//       clusters of close eigenvalues, which inverse iteration alone does
//       not separate);
//   (4) back-transformation Z = H Y, 16 lanes per vector.
// Eigenvalues ascending into ev[0..nsel), eigenvectors into Z's columns
// 0..nsel-1 (ld).  work: 3 n nsel doubles; sw: 4 ld + blockDim + 3 nsel
// doubles (shared memory); nsel <= 16, blockDim >= 16 nsel.  The eigenvalues
// are accurate to a few units of roundoff times ||A||, the vectors
// orthonormal to roundoff.
__device__ void tridiag_lowest_cta(double *A, double *Z, int n, int ld, int nsel, double *ev,
                                   double *work, double *sw) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  double *sd = sw, *se = sw + ld, *sg = sw + 2 * ld, *sp = sw + 3 * ld;
  double *sx = sw + 4 * ld;            // [nt] per-thread scratch (counts, dots)
  double *slo = sx + nt, *shi = slo + nsel, *sdt = shi + nsel;   // [nsel] each
  __shared__ double s_lohi[3];   // Gershgorin bounds, pivot floor
  __shared__ int s_open[2];   // intervals still open, by round parity
  // (1) tridiagonalisation
  for (int k = 0; k + 2 < n; ++k) {
    const int len = n - k - 1;
    if (warp == 0) {
      double sig = 0.0;
      for (int i = lane; i < len; i += 32) {
        const double x = A[(k + 1 + i) * ld + k];
        sig += x * x;
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) sig += __shfl_xor_sync(0xffffffffu, sig, o);
      if (lane == 0) {
        const double x0 = A[(k + 1) * ld + k];
        if (sig - x0 * x0 <= 1e-300 * fmax(1.0, sig)) {   // column already reduced
          se[k] = x0;
          sg[k] = 0.0;
        } else {
          const double alpha = -copysign(sqrt(sig), x0);
          se[k] = alpha;
          sg[k] = 1.0 / (sig - x0 * alpha);                 // 2 / v^T v
          A[(k + 1) * ld + k] = x0 - alpha;                 // v = x - alpha e_1
        }
      }
    }
    __syncthreads();
    const double g = sg[k];
    if (g == 0.0) continue;                                  // uniform
    // p = g A_sub v, 8 lanes per row
    for (int i0 = 0; i0 < len; i0 += nt / 8) {
      const int i = i0 + tid / 8, sub = tid & 7;
      double acc = 0.0;
      if (i < len) {
        const double *row = A + (k + 1 + i) * ld + (k + 1);
        for (int j = sub; j < len; j += 8) acc += row[j] * A[(k + 1 + j) * ld + k];
      }
      acc += __shfl_xor_sync(0xffffffffu, acc, 1);
      acc += __shfl_xor_sync(0xffffffffu, acc, 2);
      acc += __shfl_xor_sync(0xffffffffu, acc, 4);
      if (i < len && sub == 0) sp[i] = g * acc;
    }
    __syncthreads();
    // A_sub -= v q^T + q v^T, q = p - K v, K = g (v^T p) / 2 (each warp sums it)
    double K = 0.0;
    for (int j = lane; j < len; j += 32) K += A[(k + 1 + j) * ld + k] * sp[j];
#pragma unroll
    for (int o = 16; o; o >>= 1) K += __shfl_xor_sync(0xffffffffu, K, o);
    K *= 0.5 * g;
    for (int e = tid; e < len * len; e += nt) {
      const int i = e / len, j = e - i * len;
      const double vi = A[(k + 1 + i) * ld + k], vj = A[(k + 1 + j) * ld + k];
      A[(k + 1 + i) * ld + (k + 1 + j)] += 2.0 * K * vi * vj - vi * sp[j] - sp[i] * vj;
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) {
    sd[i] = A[i * ld + i];
    if (i == n - 2) se[i] = A[(n - 1) * ld + (n - 2)];
    if (i >= n - 2) sg[i] = 0.0;
  }
  __syncthreads();
  if (tid == 0) {
    double lo = 1e300, hi = -1e300, emax = 0.0;
    for (int i = 0; i < n; ++i) {
      const double r = (i > 0 ? fabs(se[i - 1]) : 0.0) + (i + 1 < n ? fabs(se[i]) : 0.0);
      lo = fmin(lo, sd[i] - r);
      hi = fmax(hi, sd[i] + r);
      if (i + 1 < n) emax = fmax(emax, se[i] * se[i]);
    }
    const double w = hi - lo;
    s_lohi[0] = lo - 1e-14 * w - 1e-300;
    s_lohi[1] = hi + 1e-14 * w + 1e-300;
    s_lohi[2] = 1e-290 * fmax(1.0, emax);
  }
  for (int i = tid; i + 1 < n; i += nt) sp[i] = se[i] * se[i];   // e_i^2
  __syncthreads();
  // (2) bisection, all eigenvalues at once
  const double pivmin = s_lohi[2];
  const int L = min(32, nt / nsel);
  const int grp = tid / L, lt = tid - grp * L;
  if (tid < nsel) {
    slo[tid] = s_lohi[0];
    shi[tid] = s_lohi[1];
  }
  __syncthreads();
  for (int round = 0; round < 64; ++round) {
    if (grp < nsel) {
      const double lo = slo[grp], hi = shi[grp];
      const double x = lo + double(lt + 1) * ((hi - lo) / double(L + 1));
      double q = sd[0] - x;
      int c = q < 0.0;
      for (int i = 1; i < n; ++i) {
        if (fabs(q) < pivmin) q = -pivmin;
        q = (sd[i] - x) - sp[i - 1] / q;
        c += q < 0.0;
      }
      sx[tid] = double(c);
    }
    if (round == 0 && tid == 0) s_open[0] = 0;
    __syncthreads();
    if (tid == 0) s_open[(round + 1) & 1] = 0;   // last read a round ago
    if (tid < nsel) {
      const int j = tid;
      const double lo = slo[j], hi = shi[j], step = (hi - lo) / double(L + 1);
      int l = L;
      for (int t = 0; t < L; ++t)
        if (sx[j * L + t] >= double(j + 1)) {
          l = t;
          break;
        }
      const double nlo = l > 0 ? lo + double(l) * step : lo;
      const double nhi = l < L ? lo + double(l + 1) * step : hi;
      slo[j] = nlo;
      shi[j] = nhi;
      if (nhi - nlo > 4.440892098500626e-16 * fmax(fabs(nlo), fabs(nhi)) + 1e-300)
        atomicAdd(&s_open[round & 1], 1);
    }
    __syncthreads();
    if (s_open[round & 1] == 0) break;                        // uniform
  }
  if (tid < nsel) ev[tid] = 0.5 * (slo[tid] + shi[tid]);
  __syncthreads();
  // (3) inverse iteration, one thread per eigenvalue, vector in Z's column j
  if (tid < nsel) {
    const int j = tid;
    double *dg = work + 3 * n * j, *su = dg + n, *su2 = su + n;
    double tn = 0.0;
    for (int i = 0; i < n; ++i) tn = fmax(tn, fmax(fabs(sd[i]), i + 1 < n ? fabs(se[i]) : 0.0));
    const double tiny = 2.220446049250313e-16 * fmax(tn, 1e-300);
    const double lam = ev[j];
    for (int i = 0; i < n; ++i)
      Z[i * ld + j] = double((uint32_t(j + 1) * 2654435761u + uint32_t(i) * 40503u) % 1000u) / 1000.0 + 0.5;
    for (int it = 0; it < 2; ++it) {
      for (int i = 0; i < n; ++i) {
        dg[i] = sd[i] - lam;
        su[i] = i + 1 < n ? se[i] : 0.0;
        su2[i] = 0.0;
      }
      for (int i = 0; i + 1 < n; ++i) {
        const double b = se[i];
        double *y = Z + j;
        if (fabs(b) > fabs(dg[i])) {          // interchange rows i and i + 1
          const double r0 = b, r1 = dg[i + 1], r2 = su[i + 1];
          const double s0 = dg[i], s1 = su[i];
          dg[i] = r0;
          su[i] = r1;
          su2[i] = r2;
          const double t = y[i * ld];
          y[i * ld] = y[(i + 1) * ld];
          y[(i + 1) * ld] = t;
          const double mlt = s0 / r0;
          dg[i + 1] = s1 - mlt * r1;
          su[i + 1] = -mlt * r2;
          y[(i + 1) * ld] -= mlt * y[i * ld];
        } else {
          const double piv = dg[i] != 0.0 ? dg[i] : tiny;
          dg[i] = piv;
          const double mlt = b / piv;
          dg[i + 1] -= mlt * su[i];
          y[(i + 1) * ld] -= mlt * y[i * ld];
        }
      }
      if (dg[n - 1] == 0.0) dg[n - 1] = tiny;
      double nrm = 0.0;
      for (int i = n - 1; i >= 0; --i) {
        double sacc = Z[i * ld + j];
        if (i + 1 < n) sacc -= su[i] * Z[(i + 1) * ld + j];
        if (i + 2 < n) sacc -= su2[i] * Z[(i + 2) * ld + j];
        const double x = sacc / (dg[i] != 0.0 ? dg[i] : tiny);
        Z[i * ld + j] = x;
        nrm += x * x;
      }
      const double inv = rsqrt(fmax(nrm, 1e-300));
      for (int i = 0; i < n; ++i) Z[i * ld + j] *= inv;
    }
  }
  __syncthreads();
  // classical Gram-Schmidt, twice per vector, in ascending order: warp w
  // forms the coefficients against vectors i = w, w + 8, ..., all threads
  // subtract, warp 0 normalises
  for (int j = 1; j < nsel; ++j) {
    for (int pass = 0; pass < 2; ++pass) {
      for (int i = warp; i < j; i += nt / 32) {
        double dt = 0.0;
        for (int r = lane; r < n; r += 32) dt += Z[r * ld + i] * Z[r * ld + j];
#pragma unroll
        for (int o = 16; o; o >>= 1) dt += __shfl_xor_sync(0xffffffffu, dt, o);
        if (lane == 0) sdt[i] = dt;
      }
      __syncthreads();
      for (int r = tid; r < n; r += nt) {
        double v = Z[r * ld + j];
        for (int i = 0; i < j; ++i) v -= sdt[i] * Z[r * ld + i];
        Z[r * ld + j] = v;
      }
      __syncthreads();
    }
    if (warp == 0) {
      double nr = 0.0;
      for (int r = lane; r < n; r += 32) nr += Z[r * ld + j] * Z[r * ld + j];
#pragma unroll
      for (int o = 16; o; o >>= 1) nr += __shfl_xor_sync(0xffffffffu, nr, o);
      const double inv = rsqrt(fmax(nr, 1e-300));
      for (int r = lane; r < n; r += 32) Z[r * ld + j] *= inv;
    }
    __syncthreads();
  }
  // (4) Z = H Y: reflectors applied last first, 16 lanes per vector
  {
    const int c = tid >> 4, l16 = tid & 15;
    const bool live = c < nsel;
    for (int k = n - 3; k >= 0; --k) {
      const double g = sg[k];
      if (g == 0.0) continue;                                // uniform
      double dt = 0.0;
      if (live)
        for (int r = k + 1 + l16; r < n; r += 16) dt += A[r * ld + k] * Z[r * ld + c];
#pragma unroll
      for (int o = 8; o; o >>= 1) dt += __shfl_xor_sync(0xffffffffu, dt, o);
      dt *= g;
      if (live)
        for (int r = k + 1 + l16; r < n; r += 16) Z[r * ld + c] -= dt * A[r * ld + k];
      __syncwarp();
    }
  }
  __syncthreads();
}

// Rayleigh-Ritz on span[X W P] by SVQB: with D the diagonal scaling of the
// basis Gram B, eigendecompose D B D = U S U^T, drop directions with
// S < tau max(S) (near-dependent or null columns, e.g. a preconditioned
// residual that is almost parallel to X), Q = U_keep S_keep^-1/2, then solve
// the standard problem (Q^T D A D Q) z = theta z and return Y = D Q Z.
template <int B>
__global__ void __launch_bounds__(256)
rr_kernel(DotState *st, const double *partial, const double *norms, double *theta,
          double *coef, double *relres, RRParams prm) {
  constexpr int m = 3 * B;
  extern __shared__ double sm[];
  double *sA = sm;             // m*m
  double *sB = sA + m * m;     // m*m
  double *sT = sB + m * m;     // m*m
  double *sZ = sT + m * m;     // m*m
  double *sD = sZ + m * m;     // m    column scaling
  double *sE = sD + m;         // m    eigenvalues
  double *sR = sE + m;         // B    relative residuals
  double *sW = sR + B;         // 4m + 256 + 3B  scratch of the tridiagonal eigensolver
  __shared__ int s_flag, s_r, s_keep[kMaxM], s_sel[kMaxM];
  __shared__ double s_red[256];
  __shared__ double s_c[kMaxM / 2 + 1], s_s[kMaxM / 2 + 1];
  __shared__ int s_p[kMaxM / 2 + 1], s_q[kMaxM / 2 + 1];

  const int d = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  DotState &s = st[d];
  if (!s.active) return;
  double *th = theta + size_t(d) * B;
  if (tid == 0) s_flag = 0;
  __syncthreads();

  // 1. convergence test on the residual norms of the current X.
  // rel_j = ||r_j|| / (|theta_j| ||M x_j||) is reported; the stopping rule is
  // the quadratic eigenvalue-error estimate
  //   est_j = kSafety (||r_j|| / ||M x_j||)^2 / ((theta_{B-1} - theta_j) |theta_j|)
  // (residual squared over the gap to the block edge, relative to |theta_j|;
  // kSafety covers ||r||_{M^-1} exceeding ||r|| / ||M x|| for residuals in the
  // high modes of M).
  if (s.have_res) {
    // chunk sums of the residual norms: 8 fixed groups of chunks per column,
    // then the groups in order
    {
      const int col = tid % B, grpc = tid / B;
      if (grpc < 8) {
        double rr = 0.0, mx = 0.0;
        for (int c = s.chunk0 + grpc; c < s.chunk1; c += 8) {
          rr += norms[size_t(c) * 2 * B + col];
          mx += norms[size_t(c) * 2 * B + B + col];
        }
        sW[grpc * 2 * B + col] = rr;
        sW[grpc * 2 * B + B + col] = mx;
      }
    }
    __syncthreads();
    if (tid < B) {
      double rr = 0.0, mx = 0.0;
      for (int g = 0; g < 8; ++g) {
        rr += sW[g * 2 * B + tid];
        mx += sW[g * 2 * B + B + tid];
      }
      const double at = fmax(fmax(fabs(th[tid]), prm.eig_scale), 1e-300);
      const double ares = sqrt(rr / fmax(mx, 1e-300));
      const double gap = fmax(th[B - 1] - th[tid], 1e-300);
      const double rel = ares / at;
      double est = kSafety * ares * ares / (gap * at);
      if (!isfinite(est)) est = 1e300;
      sE[tid] = est;                               // uncapped, for the stagnation test
      sR[tid] = (rel <= kRelCap) ? est : 1e300;
      relres[size_t(d) * B + tid] = rel;
    }
    __syncthreads();
    if (tid == 0) {
      double worst = 0.0, worst_raw = 0.0;
      for (int j = 0; j < prm.k; ++j) {
        worst = fmax(worst, sR[j]);
        worst_raw = fmax(worst_raw, sE[j]);
      }
      const bool ph32 = s.phase == 0;
      int stop = 0;
      if (worst <= (ph32 ? prm.tol32 : prm.tol)) {
        stop = 1;
        if (!ph32) s.status = 1;
      } else if (ph32) {
        if (worst_raw < 0.5 * s.best) {
          s.best = worst_raw;
          s.stag = 0;
        } else if (++s.stag >= prm.stag_window) {
          stop = 1;
        }
      }
      if (!stop && s.iters >= prm.max_iter) {
        stop = 1;
        if (!ph32) s.status = 3;
      }
      if (stop) {
        if (ph32) {          // hand over to the FP64 phase
          s.run[0] = 0;
          s.switching = 1;
        } else {
          s.active = 0;
          s.run[1] = 0;
        }
        s_flag = 1;
      }
    }
    __syncthreads();
    if (s_flag) return;
  }

  // Jacobi threshold: the FP32 phase's Gram matrices carry ~1e-7 relative
  // errors, so resolving the small eigenproblems beyond 1e-10 buys nothing
  // (and the mixed form's finishing phase carries FP32 W and P blocks: below
  // 1e-12 their rounding is all a rotation would resolve)
  const double jrel = s.phase == 0 ? kJacobiRel32 : (prm.mixed ? kJacobiRelMx : kJacobiRel64);

  // 2. Gram matrices of the dot (summed over its chunks by dot_reduce_kernel)
  const double *gsum = partial + size_t(d) * 2 * m * m;
  for (int idx = tid; idx < m * m; idx += nt) {
    sT[idx] = gsum[idx];
    sZ[idx] = gsum[m * m + idx];
  }
  __syncthreads();
  const bool has_p = s.has_p != 0;
  if (tid < m) {
    const double bii = sZ[tid * m + tid];
    const bool use = (has_p || tid < 2 * B) && bii > 0.0 && isfinite(bii);
    sD[tid] = use ? rsqrt(bii) : 0.0;
  }
  __syncthreads();
  for (int idx = tid; idx < m * m; idx += nt) {
    const int i = idx / m, j = idx % m;
    const double dd = sD[i] * sD[j];
    sA[idx] = 0.5 * (sT[i * m + j] + sT[j * m + i]) * dd;
    sB[idx] = 0.5 * (sZ[i * m + j] + sZ[j * m + i]) * dd;
  }
  __syncthreads();
  // 3. Orthonormal basis of span[X W P] in the scaled B-inner product, as
  //    Q (m x r) in sT.  FP32 phase: Cholesky B' = L L^T (outer-product form,
  //    one barrier per column) and Q = L^-T, as long as every pivot stays above
  //    kCholPivot32 (the scaled Gram has a unit diagonal, so a pivot is the
  //    squared distance of a basis vector from the span of the previous ones);
  //    likewise in the mixed form's finishing phase above kCholPivotMx.
  //    Otherwise, and always in the plain FP64 form: SVQB (Jacobi on B', drop
  //    directions with S < tau max S, Q = U_keep S_keep^-1/2).
  bool chol = false;
  if (s.phase == 0 || prm.mixed) {
    const double pivot_floor = s.phase == 0 ? kCholPivot32 : kCholPivotMx;
    const int mu = has_p ? m : 2 * B;
    bool usable = true;
    for (int i = 0; i < mu; ++i) usable = usable && sD[i] > 0.0;
    if (usable) {
      for (int idx = tid; idx < m * m; idx += nt) sZ[idx] = sB[idx];
      __syncthreads();
      // A direction of P whose pivot falls below the floor lies within
      // sqrt(floor) of the span of the columns before it: it is dropped (its
      // column takes no part in the elimination); a small pivot of X or W
      // sends the basis to SVQB.
      bool ok = true;
      int r = 0;   // kept columns, in order, in s_keep
      for (int k = 0; k < mu; ++k) {
        const double piv = sZ[k * m + k];   // final since the previous barrier
        if (!(piv > pivot_floor)) {         // every thread reads the same value
          if (k >= 2 * B) continue;
          ok = false;
          break;
        }
        if (tid == 0) s_keep[r] = k;
        ++r;
        const double ip = 1.0 / piv;
        const int R = mu - k - 1;
        for (int idx = tid; idx < R * R; idx += nt) {
          const int i = k + 1 + idx / R, j = k + 1 + idx % R;
          if (j <= i) sZ[i * m + j] -= sZ[i * m + k] * sZ[j * m + k] * ip;
        }
        __syncthreads();
      }
      if (ok) {
        __syncthreads();   // s_keep complete
        // L of the kept columns (r x r): L[c][c] = sqrt(piv), L[i][c] =
        // Z[K_i][K_c] / sqrt(piv_c) into sT; 1/L[c][c] in sE
        if (tid < r) sE[tid] = rsqrt(sZ[s_keep[tid] * m + s_keep[tid]]);
        __syncthreads();
        for (int idx = tid; idx < r * r; idx += nt) {
          const int i = idx / r, c = idx % r;
          if (c < i) sT[i * m + c] = sZ[s_keep[i] * m + s_keep[c]] * sE[c];
        }
        __syncthreads();
        // L^-1 (lower) into sB, one column per thread
        if (tid < r) {
          const int j = tid;
          for (int i = 0; i < j; ++i) sB[i * m + j] = 0.0;
          sB[j * m + j] = sE[j];
          for (int i = j + 1; i < r; ++i) {
            double sum = 0.0;
            for (int l = j; l < i; ++l) sum += sT[i * m + l] * sB[l * m + j];
            sB[i * m + j] = -sum * sE[i];
          }
        }
        __syncthreads();
        // Q = L^-T on the kept rows (m x r; dropped and unused rows zero)
        for (int idx = tid; idx < m * m; idx += nt) sT[idx] = 0.0;
        __syncthreads();
        for (int idx = tid; idx < r * r; idx += nt) {
          const int i = idx / r, c = idx % r;
          if (c >= i) sT[s_keep[i] * m + c] = sB[c * m + i];
        }
        if (tid == 0) s_r = r;
        __syncthreads();
        chol = true;
      } else {
        __syncthreads();
      }
    }
  }
  if (!chol) {
    jacobi_cta(sB, sZ, m, m, jrel, s_red, s_c, s_s, s_p, s_q);
    if (tid == 0) {
      double smax = 0.0;
      for (int i = 0; i < m; ++i) smax = fmax(smax, sB[i * m + i]);
      const double tau = s.phase == 0 ? QD_SVQB_TAU32 : QD_SVQB_TAU64;
      int r = 0;
      for (int i = 0; i < m; ++i)
        if (sB[i * m + i] > tau * smax && smax > 0.0) s_keep[r++] = i;
      s_r = r;
    }
    __syncthreads();
    const int r = s_r;
    if (r < B || !(r > 0)) {
      if (tid == 0) {
        s.active = 0;
        s.run[0] = s.run[1] = 0;
        s.status = 2;
      }
      return;
    }
    // Q = U_keep S_keep^-1/2 (m x r) into sT
    for (int idx = tid; idx < m * m; idx += nt) {
      const int i = idx / m, c = idx % m;
      double q = 0.0;
      if (c < r) {
        const int kc = s_keep[c];
        q = sZ[i * m + kc] * rsqrt(sB[kc * m + kc]);
      }
      sT[idx] = q;
    }
    __syncthreads();
  }
  const int r = s_r;
  // sZ = A' Q (m x r);  sB = Q^T sZ (r x r)
  for (int idx = tid; idx < m * r; idx += nt) {
    const int i = idx / r, c = idx % r;
    double sum = 0.0;
    for (int l = 0; l < m; ++l) sum += sA[i * m + l] * sT[l * m + c];
    sZ[i * m + c] = sum;
  }
  __syncthreads();
  for (int idx = tid; idx < r * r; idx += nt) {
    const int i = idx / r, j = idx % r;
    double sum = 0.0;
    for (int l = 0; l < m; ++l) sum += sT[l * m + i] * sZ[l * m + j];
    sB[i * m + j] = sum;
  }
  __syncthreads();
  for (int idx = tid; idx < r * r; idx += nt) {
    const int i = idx / r, j = idx % r;
    if (i < j) {
      const double v = 0.5 * (sB[i * m + j] + sB[j * m + i]);
      sB[i * m + j] = v;
      sB[j * m + i] = v;
    }
  }
  __syncthreads();
  // 4. the B lowest eigenpairs of the standard problem of size r: values
  //    ascending into sE, vectors into sA's first B columns (sZ is free
  //    scratch now)
  tridiag_lowest_cta(sB, sA, r, m, B, sE, sZ, sW);
  if (tid < B) s_sel[tid] = tid;
  __syncthreads();
  // 5. Y = D Q Z[:, sel]  (m x B)
  double *Y = coef + size_t(d) * m * B;
  for (int idx = tid; idx < m * B; idx += nt) {
    const int i = idx / B, c = idx % B;
    const int zc = s_sel[c];
    double sum = 0.0;
    for (int l = 0; l < r; ++l) sum += sT[i * m + l] * sA[l * m + zc];
    Y[idx] = sD[i] * sum;
  }
  if (tid < B) th[tid] = sE[s_sel[tid]];
  __syncthreads();
  if (tid == 0) {
    s.has_p = 1;
    s.iters++;
    s.iters_phase++;
    if (s.phase == 0) s.iters32++;
    s.have_res = 1;
  }
}

// ---------------------------------------------------------------------------
// Update: X = S Y, P = [W P] Y_wp, HX/HP/MX/MP likewise; W = HX - MX Theta
// ---------------------------------------------------------------------------

// X = S Y, P = [W P] Y_wp  (S = [X W P]); products are recomputed explicitly
// at the start of the next iteration.  X, W, P stream through a bulk-copy
// pipeline; each thread produces (row, column) outputs of a sub-tile.
template <typename TV, int B> using UpdPipe = qd::BlockPipe<TV, B, 3, (sizeof(TV) == 8 ? 32 : 64), 4>;

template <typename TV, int B>
__global__ void __launch_bounds__(256)
update_kernel(const Chunk *chunks, const DotState *st, const double *coef, TV *X, const TV *W,
              TV *P, int *wait_err) {
  constexpr int m = 3 * B;
  using PP = UpdPipe<TV, B>;
  using ACC = TV;   // FP32 arithmetic in the FP32 phase, FP64 in the FP64 phase
  extern __shared__ __align__(128) unsigned char dsm[];
  ACC *sY = reinterpret_cast<ACC *>(dsm + PP::BYTES);
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].run[sizeof(TV) == 8]) return;
  const int tid = threadIdx.x;
  if (tid == 0 && blockIdx.x == st[ch.dot].chunk0)
    const_cast<DotState *>(st)[ch.dot].launches[sizeof(TV) == 8][2]++;
  const double *Yg = coef + size_t(ch.dot) * m * B;
  for (int i = tid; i < m * B; i += blockDim.x) sY[i] = ACC(Yg[i]);
  const TV *src[3] = {X, W, P};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);   // its barrier also publishes sY
  // Elements step by a multiple of B, so each thread keeps one column j and
  // holds that column of Y in registers (threads past the multiple idle).
  const int nthr = (int(blockDim.x) / B) * B;
  const int j = tid % B;
  const bool owner = tid < nthr;
  ACC cy[3 * B];
#pragma unroll
  for (int q = 0; q < 3 * B; ++q) cy[q] = sY[q * B + j];
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (ok && owner) {
      const int nr = pipe.rows(i), r0 = pipe.row0(i);
      const TV *tx = pipe.tile(i, 0), *tw = pipe.tile(i, 1), *tp = pipe.tile(i, 2);
      for (int e = tid; e < nr * B; e += nthr) {
        const int row = e / B;
        ACC x = 0, p = 0;
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          TV t[4];
          lds4(tx + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) x = fma(ACC(t[u]), cy[q4 + u], x);
        }
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          TV t[4];
          lds4(tw + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const ACC v = ACC(t[u]) * cy[B + q4 + u];
            x += v;
            p += v;
          }
        }
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          TV t[4];
          lds4(tp + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const ACC v = ACC(t[u]) * cy[2 * B + q4 + u];
            x += v;
            p += v;
          }
        }
        const size_t o = size_t(r0) * B + e;
        X[o] = TV(x);
        P[o] = TV(p);
      }
    }
    pipe.release(i, ok);
  }
  pipe.finish(ok, wait_err);
}

// M-orthogonalisation of W against X, in memory:
//   C_W = X^T M W = (MX)^T W  (X is M-orthonormal),  W <- W - X C_W.
// Near convergence the preconditioned residual is dominated by a component
// along X and the useful correction is 1e-6..1e-8 of it; removed here by an
// elementwise subtraction it stays accurate, whereas inside the small
// Rayleigh-Ritz problem it would sit below the resolution of the Gram matrix
// and the iteration stalls.  P = [W P] Y_wp is built from directions already
// M-orthogonal to the previous X, so its component along the new X is of the
// order of |P|^2 and the Rayleigh-Ritz step resolves it.
template <typename TV, int B> using OgPipe = qd::BlockPipe<TV, B, 2, (sizeof(TV) == 8 ? 32 : 64), 4>;
template <int B> struct OgCfg {
  static constexpr int NQ = B / 4;
  static constexpr int NT = NQ * NQ;         // 4x4 output blocks of MX^T W
  static constexpr int RG = 256 / NT;        // row groups
  static constexpr size_t RED_BYTES = size_t(RG) * NT * 16 * sizeof(double);
};

// Per chunk: partial = MX^T W (B x B, FP64).  Each thread owns a 4x4 output
// block for one row group, accumulating in TV within a sub-tile and in FP64
// across sub-tiles; the row groups are summed in a fixed order.
template <typename TV, int B>
__global__ void __launch_bounds__(256)
ortho_gram_kernel(const Chunk *chunks, const DotState *st, const TV *MX, const TV *W,
                  double *partial, int *wait_err) {
  using PP = OgPipe<TV, B>;
  using C = OgCfg<B>;
  constexpr int NQ = C::NQ, NT = C::NT, RG = C::RG, NOUT = B * B;
  extern __shared__ __align__(128) unsigned char dsm[];
  double *red = reinterpret_cast<double *>(dsm + PP::BYTES);
  const Chunk ch = chunks[blockIdx.x];
  const DotState &sd = st[ch.dot];
  if (!sd.run[sizeof(TV) == 8]) return;
  const int tid = threadIdx.x;
  const bool worker = tid < NT * RG;
  const int task = tid % NT, rg = tid / NT;
  const int bi = task / NQ, bj = task % NQ;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  const TV *src[2] = {MX, W};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (ok && worker) {
      const int nr = pipe.rows(i);
      const TV *tm = pipe.tile(i, 0) + 4 * bi, *tr = pipe.tile(i, 1) + 4 * bj;
      TV t[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) t[a][b] = TV(0);
      for (int row = rg; row < nr; row += RG) {
        TV x[4], y[4];
        lds4(tm + row * B, x);
        lds4(tr + row * B, y);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) t[a][b] = fma(x[a], y[b], t[a][b]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += double(t[a][b]);
    }
    pipe.release(i, ok);
  }
  if (!pipe.finish(ok, wait_err)) return;
  if (worker) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) red[(size_t(rg) * NT + task) * 16 + a * 4 + b] = acc[a][b];
  }
  __syncthreads();
  double *out = partial + size_t(blockIdx.x) * NOUT;
  for (int e = tid; e < NOUT; e += blockDim.x) {
    const int i = e / B, j = e % B;
    const int tk = (i / 4) * NQ + (j / 4), ab = (i % 4) * 4 + (j % 4);
    double v = 0.0;
    for (int g = 0; g < RG; ++g) v += red[(size_t(g) * NT + tk) * 16 + ab];
    out[e] = v;
  }
}

// W <- W - X C_W.
template <typename TV, int B> using OaPipe = qd::BlockPipe<TV, B, 2, (sizeof(TV) == 8 ? 32 : 64), 4>;

template <typename TV, int B>
__global__ void __launch_bounds__(256)
ortho_apply_kernel(const Chunk *chunks, const DotState *st, const double *csum, const TV *X,
                   TV *W, int *wait_err) {
  using PP = OaPipe<TV, B>;
  constexpr int NOUT = B * B;
  extern __shared__ __align__(128) unsigned char dsm[];
  TV *sC = reinterpret_cast<TV *>(dsm + PP::BYTES);
  const Chunk ch = chunks[blockIdx.x];
  const DotState &sd = st[ch.dot];
  if (!sd.run[sizeof(TV) == 8]) return;
  const int tid = threadIdx.x;
  for (int e = tid; e < NOUT; e += blockDim.x) sC[e] = TV(csum[size_t(ch.dot) * NOUT + e]);
  const TV *src[2] = {X, W};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);   // its barrier also publishes sC
  // Elements step by a multiple of B, so each thread keeps one column j and
  // holds that column of C_W in registers (threads past the multiple idle).
  const int nthr = (int(blockDim.x) / B) * B;
  const int j = tid % B;
  const bool owner = tid < nthr;
  TV cw[B];
#pragma unroll
  for (int q = 0; q < B; ++q) cw[q] = sC[q * B + j];
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (ok && owner) {
      const int nr = pipe.rows(i), r0 = pipe.row0(i);
      const TV *tx = pipe.tile(i, 0), *tw = pipe.tile(i, 1);
      for (int e = tid; e < nr * B; e += nthr) {
        const int row = e / B;
        TV dw = 0;
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          TV t[4];
          lds4(tx + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) dw = fma(t[u], cw[q4 + u], dw);
        }
        W[size_t(r0) * B + e] = tw[e] - dw;
      }
    }
    pipe.release(i, ok);
  }
  pipe.finish(ok, wait_err);
}

// ---------------------------------------------------------------------------
// The mixed form's finishing phase: X, HX, MX in FP64 (the residual, the
// Rayleigh-Ritz blocks of X and the update of X carry the 1e-9 target), the
// search directions W, P and their products HW, HP, MW, MP in FP32 (the
// blocks whose rounding enters the Ritz values only through their small
// coefficients).  The kernels below are the mixed-type forms of the FP32/FP64
// ones above; all arithmetic on FP64 data is FP64.
// ---------------------------------------------------------------------------

// Per chunk: partial = [MX^T W, MX^T P] (B x B each) with FP64 MX and FP32 W, P.
template <int B> using OgMxPipe = qd::MixedPipe<double, 1, float, 1, B, 32, 4>;

template <int B>
__global__ void __launch_bounds__(256)
ortho_gram_mx_kernel(const Chunk *chunks, const DotState *st, const double *MX, const float *W,
                     double *partial, int *wait_err) {
  using PP = OgMxPipe<B>;
  using C = OgCfg<B>;
  constexpr int NQ = C::NQ, NT = C::NT, RG = C::RG, NOUT = B * B;
  extern __shared__ __align__(128) unsigned char dsm[];
  double *red = reinterpret_cast<double *>(dsm + PP::BYTES);
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].run[1]) return;
  const int tid = threadIdx.x;
  const bool worker = tid < NT * RG;
  const int task = tid % NT, rg = tid / NT;
  const int bi = task / NQ, bj = task % NQ;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  const void *src[2] = {MX, W};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (ok && worker) {
      const int nr = pipe.rows(i);
      const double *tm = pipe.tx(i, 0) + 4 * bi;
      const float *tr = pipe.tw(i, 0) + 4 * bj;
      for (int row = rg; row < nr; row += RG) {
        double x[4];
        float y[4];
        lds4(tm + row * B, x);
        lds4(tr + row * B, y);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], double(y[b]), acc[a][b]);
      }
    }
    pipe.release(i, ok);
  }
  if (!pipe.finish(ok, wait_err)) return;
  if (worker) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) red[(size_t(rg) * NT + task) * 16 + a * 4 + b] = acc[a][b];
  }
  __syncthreads();
  double *out = partial + size_t(blockIdx.x) * NOUT;
  for (int e = tid; e < NOUT; e += blockDim.x) {
    const int i = e / B, j = e % B;
    const int tk = (i / 4) * NQ + (j / 4), ab = (i % 4) * 4 + (j % 4);
    double v = 0.0;
    for (int g = 0; g < RG; ++g) v += red[(size_t(g) * NT + tk) * 16 + ab];
    out[e] = v;
  }
}

// W <- W - X C_W, FP64 arithmetic on the exact FP32 inputs, the result
// rounded once to FP32 (relative to itself: the cancellation happens before
// the rounding).
template <int B> using OaMxPipe = qd::MixedPipe<double, 1, float, 1, B, 32, 4>;

template <int B>
__global__ void __launch_bounds__(256)
ortho_apply_mx_kernel(const Chunk *chunks, const DotState *st, const double *csum,
                      const double *X, float *W, int *wait_err) {
  using PP = OaMxPipe<B>;
  constexpr int NOUT = B * B;
  extern __shared__ __align__(128) unsigned char dsm[];
  double *sC = reinterpret_cast<double *>(dsm + PP::BYTES);
  const Chunk ch = chunks[blockIdx.x];
  const DotState &sd = st[ch.dot];
  if (!sd.run[1]) return;
  const int tid = threadIdx.x;
  for (int e = tid; e < NOUT; e += blockDim.x) sC[e] = csum[size_t(ch.dot) * NOUT + e];
  const void *src[2] = {X, W};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);   // its barrier also publishes sC
  const int nthr = (int(blockDim.x) / B) * B;
  const int j = tid % B;
  const bool owner = tid < nthr;
  double cw[B];
#pragma unroll
  for (int q = 0; q < B; ++q) cw[q] = sC[q * B + j];
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (ok && owner) {
      const int nr = pipe.rows(i), r0 = pipe.row0(i);
      const double *tx = pipe.tx(i, 0);
      const float *tw = pipe.tw(i, 0);
      for (int e = tid; e < nr * B; e += nthr) {
        const int row = e / B;
        double dw = 0.0;
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          double t[4];
          lds4(tx + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) dw = fma(t[u], cw[q4 + u], dw);
        }
        W[size_t(r0) * B + e] = float(double(tw[e]) - dw);
      }
    }
    pipe.release(i, ok);
  }
  pipe.finish(ok, wait_err);
}

// Gram partials of the finishing phase, per chunk A_c = S^T HS, B_c = S^T MS
// for S = [X W P].  The rows of the X block are formed from the FP64
// products, (S^T HS)_{x, s} = (H x)^T s (H and M symmetric): HX^T X, HX^T W,
// HX^T P (and MX^T ...), in FP64; the W and P rows from FP32 data, summed in
// FP32 within a sub-tile and in FP64 across sub-tiles.  Same task layout and
// output as gram_kernel<double, B>.
template <int B> using GramMxPipe = qd::MixedPipe<double, 3, float, 6, B, 32, 3>;

template <int B>
__global__ void __launch_bounds__(GramCfg<double, B>::THREADS, 2)
gram_mx_kernel(const Chunk *chunks, const DotState *st, const double *X, const float *W,
               const float *P, const double *HX, const float *HW, const float *HP,
               const double *MX, const float *MW, const float *MP, double *partial,
               int *wait_err) {
  using C = GramCfg<double, B>;
  using PP = GramMxPipe<B>;
  constexpr int m = C::m, NT = C::NT, NT2 = C::NT2, RG = C::RG;
  extern __shared__ __align__(128) unsigned char dsm[];
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].run[1]) return;
  const int tid = threadIdx.x;
  if (tid == 0 && blockIdx.x == st[ch.dot].chunk0)
    const_cast<DotState *>(st)[ch.dot].launches[1][1]++;
  const bool worker = tid < NT2 * RG;
  const int task2 = tid % NT2, rg = tid / NT2;
  // tasks ordered by kind, so that the lanes of a warp share one code path:
  //   2: (W or P)^T (HW, HP, MW or MP)   bi, bj in [GB, NB)
  //   1: (HX or MX)^T (W or P)           bi in [0, GB), bj in [GB, NB)
  //   0: (HX or MX)^T X                  bi, bj in [0, GB)
  // each kind for S^T HS (which 0), then for S^T MS
  constexpr int GB = B / 4, T2 = (2 * GB) * (2 * GB + 1) / 2, T1 = GB * 2 * GB,
                T0 = GB * (GB + 1) / 2;
  static_assert(T2 + T1 + T0 == NT, "task split");
  int which, kind, bi, bj;
  {
    int t = task2, k, size, base;
    if (t < 2 * T2) {
      kind = 2; which = t / T2; k = t % T2; size = 2 * GB; base = GB;
    } else if ((t -= 2 * T2) < 2 * T1) {
      kind = 1; which = t / T1; k = t % T1; size = 0; base = 0;
    } else {
      t -= 2 * T1;
      kind = 0; which = t / T0; k = t % T0; size = GB; base = 0;
    }
    if (kind == 1) {
      bi = k / (2 * GB);
      bj = GB + k % (2 * GB);
    } else {   // upper triangle of a size x size square starting at base
      int r = 0;
      while (k >= size - r) {
        k -= size - r;
        ++r;
      }
      bi = base + r;
      bj = base + r + k;
    }
  }
  const int bs = (4 * bi) / B, br = (4 * bj) / B, cs = (4 * bi) % B, cr = (4 * bj) % B;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  // pipe blocks: FP64 X, HX, MX; FP32 W, P, HW, HP, MW, MP
  const void *src[9] = {X, HX, MX, W, P, HW, HP, MW, MP};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (worker && ok) {
      const int nr = pipe.rows(i);
      if (kind == 2) {
        const float *sa_p = pipe.tw(i, bs - 1) + cs;
        const float *rb_p = pipe.tw(i, 2 + 2 * which + (br - 1)) + cr;
        float t[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) t[a][b] = 0.f;
        for (int row = rg; row < nr; row += RG) {
          float sa[4], rb[4];
          lds4(sa_p + row * B, sa);
          lds4(rb_p + row * B, rb);
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) t[a][b] = fmaf(sa[a], rb[b], t[a][b]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] += double(t[a][b]);
      } else {
        const double *sa_p = pipe.tx(i, 1 + which) + cs;
        for (int row = rg; row < nr; row += RG) {
          double sa[4], rb[4];
          lds4(sa_p + row * B, sa);
          if (kind == 0) {
            lds4(pipe.tx(i, 0) + cr + row * B, rb);
          } else {
            float rf[4];
            lds4(pipe.tw(i, br - 1) + cr + row * B, rf);
#pragma unroll
            for (int b = 0; b < 4; ++b) rb[b] = double(rf[b]);
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = fma(sa[a], rb[b], acc[a][b]);
        }
      }
    }
    pipe.release(i, ok);
  }
  if (!pipe.finish(ok, wait_err)) return;
  double *out = partial + size_t(blockIdx.x) * 2 * m * m;
  if (RG > 1) {
    double *red = reinterpret_cast<double *>(dsm);   // NT2 * 16 doubles < one stage
    for (int g = 1; g < RG; ++g) {
      if (worker && rg == g) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) red[task2 * 16 + a * 4 + b] = acc[a][b];
      }
      __syncthreads();
      if (worker && rg == 0) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] += red[task2 * 16 + a * 4 + b];
      }
      __syncthreads();
    }
  }
  if (worker && rg == 0) {
    double *o = out + size_t(which) * m * m;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int i = 4 * bi + a, j = 4 * bj + b;
        o[i * m + j] = acc[a][b];
        if (bi != bj) o[j * m + i] = acc[a][b];
      }
  }
}

// X <- S Y in FP64 (X FP64, W and P FP32 exact in FP64); P <- [W P] Y_wp
// rounded to FP32.
template <int B> using UpdMxPipe = qd::MixedPipe<double, 1, float, 2, B, 32, 4>;

template <int B>
__global__ void __launch_bounds__(256)
update_mx_kernel(const Chunk *chunks, const DotState *st, const double *coef, double *X,
                 const float *W, float *P, int *wait_err) {
  constexpr int m = 3 * B;
  using PP = UpdMxPipe<B>;
  extern __shared__ __align__(128) unsigned char dsm[];
  double *sY = reinterpret_cast<double *>(dsm + PP::BYTES);
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].run[1]) return;
  const int tid = threadIdx.x;
  if (tid == 0 && blockIdx.x == st[ch.dot].chunk0)
    const_cast<DotState *>(st)[ch.dot].launches[1][2]++;
  const double *Yg = coef + size_t(ch.dot) * m * B;
  for (int i = tid; i < m * B; i += blockDim.x) sY[i] = Yg[i];
  const void *src[3] = {X, W, P};
  PP pipe;
  pipe.init(dsm, src, ch.begin, ch.end);   // its barrier also publishes sY
  const int nthr = (int(blockDim.x) / B) * B;
  const int j = tid % B;
  const bool owner = tid < nthr;
  double cy[3 * B];
#pragma unroll
  for (int q = 0; q < 3 * B; ++q) cy[q] = sY[q * B + j];
  bool ok = true;
  for (int i = 0; i < pipe.nsub; ++i) {
    ok = pipe.wait(i) && ok;
    if (ok && owner) {
      const int nr = pipe.rows(i), r0 = pipe.row0(i);
      const double *tx = pipe.tx(i, 0);
      const float *tw = pipe.tw(i, 0), *tp = pipe.tw(i, 1);
      for (int e = tid; e < nr * B; e += nthr) {
        const int row = e / B;
        double x = 0.0, p = 0.0;
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          double t[4];
          lds4(tx + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) x = fma(t[u], cy[q4 + u], x);
        }
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          float t[4];
          lds4(tw + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const double v = double(t[u]) * cy[B + q4 + u];
            x += v;
            p += v;
          }
        }
#pragma unroll
        for (int q4 = 0; q4 < B; q4 += 4) {
          float t[4];
          lds4(tp + row * B + q4, t);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const double v = double(t[u]) * cy[2 * B + q4 + u];
            x += v;
            p += v;
          }
        }
        const size_t o = size_t(r0) * B + e;
        X[o] = x;
        P[o] = float(p);
      }
    }
    pipe.release(i, ok);
  }
  pipe.finish(ok, wait_err);
}

// FP32 -> finishing-phase hand-over in the mixed form: X64 = X32 on the rows
// of the dots that left the FP32 phase this iteration (P, W and the products
// stay in their FP32 blocks; the first finishing iteration recomputes them).
template <int B>
__global__ void transition_x_kernel(const Chunk *chunks, const DotState *st, const float *X32,
                                    double *X) {
  const Chunk ch = chunks[blockIdx.x];
  if (!st[ch.dot].switching) return;
  for (int idx = threadIdx.x; idx < (ch.end - ch.begin) * B; idx += blockDim.x) {
    const size_t o = size_t(ch.begin) * B + idx;
    X[o] = double(X32[o]);
  }
}

// out[d][v] = sum over the chunks of dot d of partial[c * nvals + v], in chunk
// order (deterministic).  One thread per (dot, value): the latency of the
// chunk loop is hidden by the number of threads instead of being paid
// serially inside one CTA per dot.
__global__ void dot_reduce_kernel(const DotState *st, int ph, const double *__restrict__ partial,
                                  int nvals, double *__restrict__ out) {
  const int d = blockIdx.y;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const DotState &sd = st[d];
  if (!sd.run[ph] || v >= nvals) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int c = sd.chunk0;
  for (; c + 3 < sd.chunk1; c += 4) {
    a0 += partial[size_t(c) * nvals + v];
    a1 += partial[size_t(c + 1) * nvals + v];
    a2 += partial[size_t(c + 2) * nvals + v];
    a3 += partial[size_t(c + 3) * nvals + v];
  }
  for (; c < sd.chunk1; ++c) a0 += partial[size_t(c) * nvals + v];
  out[size_t(d) * nvals + v] = (a0 + a1) + (a2 + a3);
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

// Diagonal (Jacobi) preconditioner of the dots without a lattice (refined
// meshes, natural boundaries): per row d_r = max(|H_rr|, sum_{j != r} |H_rj|),
// the stiffness scale of the row (stiffness rows sum to about zero, so the
// off-diagonal sum tracks the diagonal even where the potential cancels it),
// and W_r <- W_r / d_r.
__global__ void jacobi_diag_kernel(const Chunk *chunks, const int32_t *__restrict__ rowptr,
                                   const int32_t *__restrict__ col,
                                   const double *__restrict__ H, double *__restrict__ dinv) {
  const Chunk ch = chunks[blockIdx.x];
  if (!ch.jacobi) return;
  for (int r = ch.begin + threadIdx.x; r < ch.end; r += blockDim.x) {
    double dg = 0.0, off = 0.0;
    for (int p = rowptr[r]; p < rowptr[r + 1]; ++p) {
      const double h = fabs(H[p]);
      if (col[p] == r) dg = h;
      else off += h;
    }
    const double d = fmax(dg, off);
    dinv[r] = d > 0.0 ? 1.0 / d : 1.0;
  }
}

template <typename TV, int B>
__global__ void jacobi_apply_kernel(const Chunk *chunks, const DotState *st, int ph,
                                    const double *__restrict__ dinv, TV *__restrict__ W) {
  const Chunk ch = chunks[blockIdx.x];
  if (!ch.jacobi || !st[ch.dot].run[ph]) return;
  for (int idx = threadIdx.x; idx < (ch.end - ch.begin) * B; idx += blockDim.x) {
    const size_t o = size_t(ch.begin) * B + idx;
    W[o] = TV(double(W[o]) * dinv[ch.begin + idx / B]);
  }
}

// Device-side control of the solver's WHILE graph (the loop over iteration
// blocks): counts the active dots and keeps the loop running while some dot
// is active, no bounded wait has expired and fewer than `cap` blocks have run.
// The block counter makes the loop end after at most `cap` bodies whatever
// the dots' state.  first != 0: the check before the first body (resets the
// counter); otherwise the check at the end of a body (counts that block).
__global__ void loop_control_kernel(const DotState *st, int n, int *count, int cap,
                                    const int *wait_err, cudaGraphConditionalHandle cond,
                                    int first) {
  __shared__ int s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) c += st[i].active;
  atomicAdd(&s, c);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int blocks = first ? 0 : count[1] + 1;
    count[0] = s;
    count[1] = blocks;
    const bool go = s > 0 && blocks < cap && *wait_err == 0;
    cudaGraphSetConditional(cond, go ? 1u : 0u);
  }
}

__global__ void transition_state_kernel(DotState *st, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  DotState &s = st[i];
  if (!s.switching) return;
  s.switching = 0;
  s.phase = 1;
  s.run[1] = 1;
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
  double *theta, *coef, *relres, *partial, *norms, *dotsum, *gramsum;
  int *count;
  double *slot[9];   // FP64 vector blocks X W P HX HW HP MX MW MP
  float *slot32[9];  // FP32 vector blocks (mixed precision only)
  int nchunks;
  // DST preconditioner
  void *tmp1, *tmp2;     // BF16 intermediates of the transform passes
  qd_dst_prec *desc;
  qd::GemmTile *tiles_x, *tiles_y;
  int64_t ntx, nty;
  int rows_x, rows_y;    // largest TMEM row block of the x / y passes
  const uint16_t *mats;
  int *wait_err;         // set by a kernel whose bounded wait ran out
  double *dinv;          // Jacobi preconditioner of the dots without a lattice
  int njac;              // chunks of such dots
  float2 *hm32;          // FP32 (H, M) pairs per nonzero (mixed precision only)
  int32_t *col32;        // copy of the column indices with bulk-copy slack (mixed only)
  uint16_t *pos16;       // staged position of every nonzero's column (mixed only):
  SubPlan *plan;         //   64-row sub-tiles (products of X and P), plan per sub-tile
  int spc;               //   sub-tiles per chunk
  uint16_t *pos16w;      // the same for 128-row sub-tiles (products of W)
  SubPlan *planw;
  int spcw;
  float *rs32;           // row sums of the FP32 H values, summed in FP64 (mixed only)
  int *hm_exp;           // largest binary exponents of |H| and |M| (scales 2^e of the pairs)
};

size_t rr_smem_bytes(int B) {
  const int m = 3 * B;
  return size_t(4 * m * m + 2 * m + B + 4 * m + 256 + 3 * B) * sizeof(double);
}

int carve(qd::Arena &ar, int n_dots, int64_t n_rows, int64_t nnz, int B, int nchunks,
          int chunk_rows, int64_t ntx, int64_t nty, bool mixed, bool jacobi, Layout &L) {
  const int m = 3 * B;
  L.chunks = ar.take<Chunk>(nchunks);
  L.row_off = ar.take<int32_t>(n_dots + 1);
  L.st = ar.take<DotState>(n_dots);
  L.theta = ar.take<double>(size_t(n_dots) * B);
  L.coef = ar.take<double>(size_t(n_dots) * m * B);
  L.relres = ar.take<double>(size_t(n_dots) * B);
  L.partial = ar.take<double>(size_t(nchunks) * 2 * m * m);
  L.dotsum = ar.take<double>(size_t(n_dots) * 2 * B * B);
  L.gramsum = ar.take<double>(size_t(n_dots) * 2 * m * m);
  L.norms = ar.take<double>(size_t(nchunks) * 2 * B);
  L.count = ar.take<int>(4);
  L.wait_err = ar.take<int>(1);
  // FP64 blocks: all nine in the plain form; X, HX, MX (slots 0, 3, 6) in the
  // mixed form, whose finishing phase keeps the search directions in FP32
  for (int i = 0; i < 9; ++i)
    L.slot[i] = (!mixed || i % 3 == 0) ? ar.take<double>(size_t(n_rows) * B) : nullptr;
  for (int i = 0; i < 9; ++i) L.slot32[i] = mixed ? ar.take<float>(size_t(n_rows) * B) : nullptr;
  // +slack: the FP32 SpMM rounds its bulk copies out to 16-byte boundaries
  L.hm32 = mixed ? ar.take<float2>(size_t(nnz) + 2) : nullptr;
  L.col32 = mixed ? ar.take<int32_t>(size_t(nnz) + 4) : nullptr;
  L.rs32 = mixed ? ar.take<float>(size_t(n_rows)) : nullptr;
  L.spc = (chunk_rows + 63) / 64;
  L.pos16 = mixed ? ar.take<uint16_t>(size_t(nnz) + 16) : nullptr;
  L.plan = mixed ? ar.take<SubPlan>(size_t(nchunks) * L.spc) : nullptr;
  L.spcw = (chunk_rows + 127) / 128;
  L.pos16w = mixed ? ar.take<uint16_t>(size_t(nnz) + 16) : nullptr;
  L.planw = mixed ? ar.take<SubPlan>(size_t(nchunks) * L.spcw) : nullptr;
  L.hm_exp = ar.take<int>(2);
  L.dinv = jacobi ? ar.take<double>(size_t(n_rows)) : nullptr;
  L.njac = 0;
  L.nchunks = nchunks;
  L.ntx = ntx;
  L.nty = nty;
  L.mats = nullptr;
  L.rows_x = L.rows_y = 16;
  if (ntx > 0) {
    L.tmp1 = ar.take<uint16_t>(size_t(n_rows) * B);
    L.tmp2 = ar.take<uint16_t>(size_t(n_rows) * B);
    L.desc = ar.take<qd_dst_prec>(n_dots);
    L.tiles_x = ar.take<qd::GemmTile>(ntx);
    L.tiles_y = ar.take<qd::GemmTile>(nty);
  } else {
    L.tmp1 = L.tmp2 = nullptr;
    L.desc = nullptr;
    L.tiles_x = L.tiles_y = nullptr;
  }
  return QD_OK;
}

// Some dot has no lattice (no descriptor, or nx <= 0): Jacobi preconditioning.
bool needs_jacobi(int n_dots, const qd_dst_prec *h_prec) {
  if (!h_prec) return true;
  for (int d = 0; d < n_dots; ++d)
    if (h_prec[d].nx <= 0) return true;
  return false;
}

int count_chunks(int n_dots, const int32_t *row_off, int chunk_rows) {
  int64_t c = 0;
  for (int d = 0; d < n_dots; ++d) {
    const int n = row_off[d + 1] - row_off[d];
    c += (n + chunk_rows - 1) / chunk_rows;
  }
  return int(c);
}

template <typename TV>
struct Bufs {
  TV *X, *W, *P, *HX, *HW, *HP, *MX, *MW, *MP;
  template <typename S>
  explicit Bufs(S *const *slot) {
    TV **dst[9] = {&X, &W, &P, &HX, &HW, &HP, &MX, &MW, &MP};
    for (int i = 0; i < 9; ++i) *dst[i] = reinterpret_cast<TV *>(slot[i]);
  }
};

// FP32 products of W (HW, MW) for the dots iterating in phase ph.
template <int B>
int spmm32_w(const Layout &L, const int32_t *rowptr, const float *W, float *HW, float *MW,
             int ph, cudaStream_t s) {
  constexpr size_t bytes = SpmmStage<B, 1, 128>::BYTES;
  if (smem_attr<spmm32s_kernel<B, false>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
  spmm32s_kernel<B, false><<<L.nchunks, 32 * B, bytes, s>>>(
      L.chunks, L.st, rowptr, L.col32, L.pos16w, L.planw, L.spcw, L.hm32, L.rs32, L.hm_exp,
      L.theta, W, nullptr, HW, MW, nullptr, nullptr, nullptr, nullptr, L.wait_err, ph);
  return QD_OK;
}

// Everything of one iteration up to the Rayleigh-Ritz step, for the dots in
// the phase of precision TV.
template <typename TV, int B>
int phase_sequence(const Layout &L, const Bufs<TV> &b, int n_dots, const int32_t *rowptr,
                   const int32_t *col, const double *H, const double *M, cudaStream_t s) {
  constexpr int G = B / 4;
  constexpr int PH = sizeof(TV) == 8 ? 1 : 0;
  using GC = GramCfg<TV, B>;
  qd::prof_begin(qd::PK_SPMM, s);
  const qd::MatF64 A{H, M};   // the FP64 form's values (the FP32 form stages its pairs)
  if constexpr (sizeof(TV) == 4) {
    constexpr size_t bytes = SpmmStage<B, 2, 64>::BYTES;
    if (smem_attr<spmm32s_kernel<B, true>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
    spmm32s_kernel<B, true><<<L.nchunks, 32 * B, bytes, s>>>(
        L.chunks, L.st, rowptr, L.col32, L.pos16, L.plan, L.spc, L.hm32, L.rs32, L.hm_exp,
        L.theta, b.X, b.P, b.HX, b.MX, b.HP, b.MP, b.W, L.norms, L.wait_err, 0);
  } else {
    spmm_xp_kernel<TV, TV, B><<<L.nchunks, 128 * G, 0, s>>>(L.chunks, L.st, rowptr, col, A,
                                                            L.theta, b.X, b.P, b.HX, b.MX,
                                                            b.HP, b.MP, b.W, L.norms);
  }
  qd::prof_end(qd::PK_SPMM, s);
  QD_CHECK_LAUNCH();
  if (L.ntx > 0) {
    qd::prof_begin(qd::PK_PRECOND, s);
    cudaError_t e = qd::dst_apply<TV>(L.tiles_x, L.ntx, L.rows_x, L.tiles_y, L.nty, L.rows_y,
                                      &L.st[0].run[PH], int(sizeof(DotState) / sizeof(int)),
                                      L.desc, L.row_off, L.mats, B, b.W, b.W, L.tmp1, L.tmp2,
                                      L.wait_err, s);
    qd::prof_end(qd::PK_PRECOND, s);
    if (e != cudaSuccess) return QD_ERR_CUDA;
  }
  if (L.njac > 0) {
    qd::prof_begin(qd::PK_PRECOND, s);
    jacobi_apply_kernel<TV, B><<<L.nchunks, 256, 0, s>>>(L.chunks, L.st, PH, L.dinv, b.W);
    qd::prof_end(qd::PK_PRECOND, s);
    QD_CHECK_LAUNCH();
  }
  qd::prof_begin(qd::PK_ORTHO, s);
  {
    constexpr size_t bytes = OgPipe<TV, B>::BYTES + OgCfg<B>::RED_BYTES;
    if (smem_attr<ortho_gram_kernel<TV, B>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
    ortho_gram_kernel<TV, B><<<L.nchunks, 256, bytes, s>>>(L.chunks, L.st, b.MX, b.W,
                                                           L.partial, L.wait_err);
  }
  QD_CHECK_LAUNCH();
  dot_reduce_kernel<<<dim3((B * B + 255) / 256, n_dots), 256, 0, s>>>(L.st, PH, L.partial,
                                                                     B * B, L.dotsum);
  QD_CHECK_LAUNCH();
  {
    constexpr size_t bytes = OaPipe<TV, B>::BYTES + B * B * sizeof(TV);
    if (smem_attr<ortho_apply_kernel<TV, B>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
    ortho_apply_kernel<TV, B><<<L.nchunks, 256, bytes, s>>>(L.chunks, L.st, L.dotsum, b.X,
                                                            b.W, L.wait_err);
  }
  qd::prof_end(qd::PK_ORTHO, s);
  QD_CHECK_LAUNCH();
  qd::prof_begin(qd::PK_SPMM, s);
  if constexpr (sizeof(TV) == 4) {
    if (spmm32_w<B>(L, rowptr, b.W, b.HW, b.MW, 0, s) != QD_OK) return QD_ERR_CUDA;
  } else {
    spmm_chunk_kernel<TV, B><<<L.nchunks, 64 * G, 0, s>>>(L.chunks, L.st, rowptr, col, A, b.W,
                                                          b.HW, b.MW);
  }
  qd::prof_end(qd::PK_SPMM, s);
  QD_CHECK_LAUNCH();
  qd::prof_begin(qd::PK_GRAM, s);
  if (smem_attr<gram_kernel<TV, B>>(GramPipe<TV, B>::BYTES) != cudaSuccess) return QD_ERR_CUDA;
  gram_kernel<TV, B><<<L.nchunks, GC::THREADS, GramPipe<TV, B>::BYTES, s>>>(
      L.chunks, L.st, b.X, b.W, b.P, b.HX, b.HW, b.HP, b.MX, b.MW, b.MP, L.partial, L.wait_err);
  QD_CHECK_LAUNCH();
  // the Gram sums of this phase's dots land in L.dotsum; the other phase's
  // dots are reduced by their own sequence (their partial chunks differ)
  dot_reduce_kernel<<<dim3((2 * 9 * B * B + 255) / 256, n_dots), 256, 0, s>>>(
      L.st, PH, L.partial, 2 * 9 * B * B, L.gramsum);
  qd::prof_end(qd::PK_GRAM, s);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

template <typename TV, int B>
int update_step(const Layout &L, const Bufs<TV> &b, cudaStream_t s) {
  qd::prof_begin(qd::PK_UPDATE, s);
  constexpr size_t bytes = UpdPipe<TV, B>::BYTES + 3 * B * B * sizeof(TV);
  if (smem_attr<update_kernel<TV, B>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
  update_kernel<TV, B><<<L.nchunks, 256, bytes, s>>>(L.chunks, L.st, L.coef, b.X, b.W, b.P,
                                                     L.wait_err);
  qd::prof_end(qd::PK_UPDATE, s);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

// Everything of one iteration up to the Rayleigh-Ritz step for the dots in
// the mixed form's finishing phase: X, HX, MX in FP64, W, P and their
// products in FP32 (b32), W's products by the FP32 SpMM.
template <int B>
int phase_sequence_mx(const Layout &L, const Bufs<float> &b, const Bufs<double> &x64,
                      int n_dots, const int32_t *rowptr, const int32_t *col, const double *H,
                      const double *M, cudaStream_t s) {
  constexpr int G = B / 4;
  using GC = GramCfg<double, B>;
  qd::prof_begin(qd::PK_SPMM, s);
  spmm_xp_kernel<double, float, B><<<L.nchunks, 128 * G, 0, s>>>(
      L.chunks, L.st, rowptr, col, qd::MatF64{H, M}, L.theta, x64.X, b.P, x64.HX, x64.MX, b.HP,
      b.MP, b.W, L.norms);
  qd::prof_end(qd::PK_SPMM, s);
  QD_CHECK_LAUNCH();
  if (L.ntx > 0) {
    qd::prof_begin(qd::PK_PRECOND, s);
    cudaError_t e = qd::dst_apply<float>(L.tiles_x, L.ntx, L.rows_x, L.tiles_y, L.nty, L.rows_y,
                                         &L.st[0].run[1], int(sizeof(DotState) / sizeof(int)),
                                         L.desc, L.row_off, L.mats, B, b.W, b.W, L.tmp1, L.tmp2,
                                         L.wait_err, s);
    qd::prof_end(qd::PK_PRECOND, s);
    if (e != cudaSuccess) return QD_ERR_CUDA;
  }
  if (L.njac > 0) {
    qd::prof_begin(qd::PK_PRECOND, s);
    jacobi_apply_kernel<float, B><<<L.nchunks, 256, 0, s>>>(L.chunks, L.st, 1, L.dinv, b.W);
    qd::prof_end(qd::PK_PRECOND, s);
    QD_CHECK_LAUNCH();
  }
  qd::prof_begin(qd::PK_ORTHO, s);
  {
    constexpr size_t bytes = OgMxPipe<B>::BYTES + OgCfg<B>::RED_BYTES;
    if (smem_attr<ortho_gram_mx_kernel<B>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
    ortho_gram_mx_kernel<B><<<L.nchunks, 256, bytes, s>>>(L.chunks, L.st, x64.MX, b.W,
                                                          L.partial, L.wait_err);
  }
  QD_CHECK_LAUNCH();
  dot_reduce_kernel<<<dim3((B * B + 255) / 256, n_dots), 256, 0, s>>>(L.st, 1, L.partial,
                                                                     B * B, L.dotsum);
  QD_CHECK_LAUNCH();
  {
    constexpr size_t bytes = OaMxPipe<B>::BYTES + B * B * sizeof(double);
    if (smem_attr<ortho_apply_mx_kernel<B>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
    ortho_apply_mx_kernel<B><<<L.nchunks, 256, bytes, s>>>(L.chunks, L.st, L.dotsum, x64.X,
                                                           b.W, L.wait_err);
  }
  qd::prof_end(qd::PK_ORTHO, s);
  QD_CHECK_LAUNCH();
  qd::prof_begin(qd::PK_SPMM, s);
  if (spmm32_w<B>(L, rowptr, b.W, b.HW, b.MW, 1, s) != QD_OK) return QD_ERR_CUDA;
  qd::prof_end(qd::PK_SPMM, s);
  QD_CHECK_LAUNCH();
  qd::prof_begin(qd::PK_GRAM, s);
  if (smem_attr<gram_mx_kernel<B>>(GramMxPipe<B>::BYTES) != cudaSuccess) return QD_ERR_CUDA;
  gram_mx_kernel<B><<<L.nchunks, GC::THREADS, GramMxPipe<B>::BYTES, s>>>(
      L.chunks, L.st, x64.X, b.W, b.P, x64.HX, b.HW, b.HP, x64.MX, b.MW, b.MP, L.partial,
      L.wait_err);
  QD_CHECK_LAUNCH();
  dot_reduce_kernel<<<dim3((2 * 9 * B * B + 255) / 256, n_dots), 256, 0, s>>>(
      L.st, 1, L.partial, 2 * 9 * B * B, L.gramsum);
  qd::prof_end(qd::PK_GRAM, s);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

template <int B>
int update_step_mx(const Layout &L, const Bufs<float> &b, const Bufs<double> &x64,
                   cudaStream_t s) {
  qd::prof_begin(qd::PK_UPDATE, s);
  constexpr size_t bytes = UpdMxPipe<B>::BYTES + 3 * B * B * sizeof(double);
  if (smem_attr<update_mx_kernel<B>>(bytes) != cudaSuccess) return QD_ERR_CUDA;
  update_mx_kernel<B><<<L.nchunks, 256, bytes, s>>>(L.chunks, L.st, L.coef, x64.X, b.W, b.P,
                                                    L.wait_err);
  qd::prof_end(qd::PK_UPDATE, s);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

// The iteration loop.  In mixed precision every dot starts in the FP32 phase
// and switches to the FP64 phase on its own (FP32 target reached, stagnation
// or iteration cap); both phases advance in every host iteration, so a dot's
// FP64 finish overlaps other dots' FP32 work.
template <int B>
int run_solver(const Layout &L, bool mixed, int n_dots, const int32_t *rowptr, const int32_t *col,
               const double *H, const double *M, const RRParams &prm, bool use_graphs,
               cudaStream_t s, int &iters_run) {
  Bufs<double> b64(L.slot);
  const size_t rr_smem = rr_smem_bytes(B);
  QD_CUDA_TRY(cudaFuncSetAttribute(rr_kernel<B>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(rr_smem)));
  // One LOBPCG iteration for every dot (both phases), enqueued on stream q.
  // The mixed form runs the FP32 phase's sequence for its FP32-phase dots and
  // the finishing sequence (FP64 X, FP32 search directions) for the others;
  // the plain form runs the FP64 sequence.
  auto iteration = [&](cudaStream_t q) -> int {
    int st;
    if (mixed) {
      Bufs<float> b32(L.slot32);
      if ((st = phase_sequence<float, B>(L, b32, n_dots, rowptr, col, H, M, q)) != QD_OK) return st;
      if ((st = phase_sequence_mx<B>(L, b32, b64, n_dots, rowptr, col, H, M, q)) != QD_OK)
        return st;
    } else {
      if ((st = phase_sequence<double, B>(L, b64, n_dots, rowptr, col, H, M, q)) != QD_OK)
        return st;
    }
    qd::prof_begin(qd::PK_RR, q);
    rr_kernel<B><<<n_dots, 256, rr_smem, q>>>(L.st, L.gramsum, L.norms, L.theta, L.coef,
                                              L.relres, prm);
    qd::prof_end(qd::PK_RR, q);
    QD_CHECK_LAUNCH();
    if (mixed) {
      Bufs<float> b32(L.slot32);
      if ((st = update_step<float, B>(L, b32, q)) != QD_OK) return st;
      if ((st = update_step_mx<B>(L, b32, b64, q)) != QD_OK) return st;
      transition_x_kernel<B><<<L.nchunks, 256, 0, q>>>(L.chunks, L.st, L.slot32[0], b64.X);
      QD_CHECK_LAUNCH();
      transition_state_kernel<<<(n_dots + 127) / 128, 128, 0, q>>>(L.st, n_dots);
      QD_CHECK_LAUNCH();
    } else {
      if ((st = update_step<double, B>(L, b64, q)) != QD_OK) return st;
    }
    return QD_OK;
  };
  // Iterations run in blocks of kGraphBlock.  The first block is enqueued
  // directly (it also sets every kernel's attributes).  The rest of the solve
  // is one CUDA graph: a WHILE conditional node whose body is one block of
  // iterations followed by loop_control_kernel, which counts the active dots
  // on the device and sets the loop condition; a check before the loop decides
  // whether the body runs at all.  So the whole solve runs with no host
  // round trip until it has converged (or hit max_iter, or a bounded wait
  // expired).  The graph is captured on a private stream and launched into the
  // caller's stream; kernel arguments are the same in every iteration
  // (per-dot progress lives on the device).  Where conditional graph nodes are
  // unavailable, with per-kernel timing enabled, or with graphs switched off
  // in the options, blocks are enqueued directly and the host reads the
  // active-dot count after each one.
  constexpr int kGraphBlock = 8;
  const bool graphs = use_graphs && !qd::prof_enabled();
  const int total_blocks = (prm.max_iter + kGraphBlock + kGraphBlock - 1) / kGraphBlock;
  struct GraphGuard {
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~GraphGuard() {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      if (cap) cudaStreamDestroy(cap);
    }
  } gg;
  iters_run = 0;
  for (int i = 0; i < kGraphBlock; ++i) {
    const int st = iteration(s);
    if (st != QD_OK) return st;
  }
  iters_run = kGraphBlock;
  if (total_blocks <= 1) return QD_OK;
  bool device_loop = false;
  if (graphs) {
    // WHILE graph: [check] -> WHILE(cond) { kGraphBlock iterations; control }
    cudaGraphConditionalHandle cond;
    cudaGraphNode_t pre = nullptr, loop = nullptr;
    size_t nnodes = 1;
    uint64_t body_launches = 0;
    bool ok = cudaStreamCreateWithFlags(&gg.cap, cudaStreamNonBlocking) == cudaSuccess &&
              cudaGraphCreate(&gg.graph, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&cond, gg.graph, 0, cudaGraphCondAssignDefault) ==
                  cudaSuccess;
    if (ok) {
      QD_CUDA_TRY(cudaStreamBeginCaptureToGraph(gg.cap, gg.graph, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal));
      loop_control_kernel<<<1, 256, 0, gg.cap>>>(L.st, n_dots, L.count, total_blocks - 1,
                                                 L.wait_err, cond, 1);
      const cudaError_t le = cudaGetLastError();
      cudaGraph_t g = gg.graph;
      QD_CUDA_TRY(cudaStreamEndCapture(gg.cap, &g));
      QD_CUDA_TRY(le);
      QD_LAUNCHED();
      ok = cudaGraphGetNodes(gg.graph, &pre, &nnodes) == cudaSuccess && nnodes == 1;
    }
    if (ok) {
      cudaGraphNodeParams p = {};
      p.type = cudaGraphNodeTypeConditional;
      p.conditional.handle = cond;
      p.conditional.type = cudaGraphCondTypeWhile;
      p.conditional.size = 1;
      ok = cudaGraphAddNode(&loop, gg.graph, &pre, 1, &p) == cudaSuccess;
      if (ok) {
        cudaGraph_t body = p.conditional.phGraph_out[0];
        QD_CUDA_TRY(cudaStreamBeginCaptureToGraph(gg.cap, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal));
        const uint64_t l0 = qd::g_launches.load();
        int st = QD_OK;
        for (int i = 0; i < kGraphBlock && st == QD_OK; ++i) st = iteration(gg.cap);
        if (st == QD_OK) {
          loop_control_kernel<<<1, 256, 0, gg.cap>>>(L.st, n_dots, L.count, total_blocks - 1,
                                                     L.wait_err, cond, 0);
          if (cudaGetLastError() != cudaSuccess) st = QD_ERR_CUDA;
          QD_LAUNCHED();
        }
        body_launches = qd::g_launches.load() - l0;
        const cudaError_t ce = cudaStreamEndCapture(gg.cap, &body);
        if (st != QD_OK) return st;
        QD_CUDA_TRY(ce);
        QD_CUDA_TRY(cudaGraphInstantiate(&gg.exec, gg.graph, 0));
        QD_CUDA_TRY(cudaGraphLaunch(gg.exec, s));
        int blocks = 0;
        QD_CUDA_TRY(cudaMemcpyAsync(&blocks, L.count + 1, sizeof(int), cudaMemcpyDeviceToHost,
                                    s));
        QD_CUDA_TRY(cudaStreamSynchronize(s));
        // the body's launches were counted once while it was captured
        if (blocks > 1)
          qd::g_launches.fetch_add(body_launches * uint64_t(blocks - 1),
                                   std::memory_order_relaxed);
        if (blocks == 0) qd::g_launches.fetch_sub(body_launches, std::memory_order_relaxed);
        iters_run += kGraphBlock * blocks;
        device_loop = true;
      }
    }
    if (!ok) cudaGetLastError();    // clear the error of an unsupported conditional node
  }
  if (!device_loop) {
    int host_count = n_dots;
    for (int blk = 1; blk < total_blocks; ++blk) {
      count_active_kernel<<<1, 256, 0, s>>>(L.st, n_dots, L.count);
      QD_CHECK_LAUNCH();
      QD_CUDA_TRY(cudaMemcpyAsync(&host_count, L.count, sizeof(int), cudaMemcpyDeviceToHost, s));
      QD_CUDA_TRY(cudaStreamSynchronize(s));
      if (host_count == 0) break;
      for (int i = 0; i < kGraphBlock; ++i) {
        const int st = iteration(s);
        if (st != QD_OK) return st;
      }
      iters_run += kGraphBlock;
    }
  }
  return QD_OK;
}

// Host-side record of the last set-up made in a workspace (at most
// kSetupCaches workspaces, most recent first): the tables copied to it and
// the count of nonzeros.  Read and written under g_setup_mutex.
struct SetupCache {
  const void *work = nullptr;
  size_t work_bytes = 0;
  const int32_t *rowptr = nullptr, *col = nullptr;
  int B = 0, prec = 0, chunk_rows = 0, jacobi = 0;
  int64_t ntx = 0, nty = 0;
  int32_t nnz = 0;
  std::vector<int32_t> row_off;
  std::vector<Chunk> chunks;
  std::vector<qd::GemmTile> tiles_x, tiles_y;
  std::vector<qd_dst_prec> desc;
};
constexpr int kSetupCaches = 8;
std::mutex g_setup_mutex;
std::vector<SetupCache> g_setup_caches;

SetupCache &setup_cache_for(const void *work) {
  for (size_t i = 0; i < g_setup_caches.size(); ++i)
    if (g_setup_caches[i].work == work) {
      if (i) std::swap(g_setup_caches[0], g_setup_caches[i]);
      return g_setup_caches[0];
    }
  if (int(g_setup_caches.size()) >= kSetupCaches) g_setup_caches.pop_back();
  g_setup_caches.insert(g_setup_caches.begin(), SetupCache{});
  return g_setup_caches[0];
}

template <typename T>
bool pod_equal(const std::vector<T> &a, const std::vector<T> &b) {
  return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(T)) == 0);
}

// Per-dot state at the start of a solve.  reset: rebuilt here from the chunk
// range the state already holds (the previous solve's, same chunk table);
// otherwise the host's copy is kept.  Theta, the residual norms and the wait
// flag are zeroed either way.
__global__ void state_reset_kernel(DotState *st, int n_dots, int reset, int phase0, int B,
                                   double *theta, double *relres, int *wait_err) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d == 0) *wait_err = 0;
  if (d >= n_dots) return;
  if (reset) {
    DotState y{};
    y.chunk0 = st[d].chunk0;
    y.chunk1 = st[d].chunk1;
    y.active = 1;
    y.phase = phase0;
    y.run[phase0] = 1;
    y.best = 1e300;
    if (y.chunk1 == y.chunk0) {
      y.active = 0;
      y.run[0] = y.run[1] = 0;
      y.status = 2;
    }
    st[d] = y;
  }
  for (int j = 0; j < B; ++j) {
    theta[size_t(d) * B + j] = 0.0;
    relres[size_t(d) * B + j] = 0.0;
  }
}

template <int B>
int solve_b(int32_t n_dots, const int32_t *h_row_off, const int32_t *d_rowptr,
            const int32_t *d_col, const double *d_H, const double *d_M,
            const qd_dst_prec *h_prec, const uint16_t *d_mats, int k, int prec_mode,
            double tol, int max_iter, uint64_t seed, double *d_X_out, double *d_E_out,
            double *d_res_out, int32_t *d_iters_out, int32_t *h_info, int32_t *h_counts,
            void *d_work, size_t work_bytes, const qd_lobpcg_opts *opts, cudaStream_t s) {
  const int64_t n_rows = h_row_off[n_dots];
  const int chunk_rows = chunk_rows_of(opts);
  const int nchunks = count_chunks(n_dots, h_row_off, chunk_rows);
  int64_t ntx = 0, nty = 0;
  if (h_prec) {
    if (!d_mats) return QD_ERR_INVALID;
    for (int d = 0; d < n_dots; ++d) {
      const qd_dst_prec &q = h_prec[d];
      if (q.nx <= 0) continue;
      if (q.ny <= 0 || int64_t(q.nx) * q.ny != h_row_off[d + 1] - h_row_off[d] ||
          q.sx_off < 0 || q.sy_off < 0 || q.sx_off % 8 || q.sy_off % 8 || !(q.cx > 0.f) ||
          !(q.cy > 0.f) || !(q.shift >= 0.f))
        return QD_ERR_INVALID;
    }
    qd::dst_tiles(n_dots, h_prec, B, nullptr, &ntx, nullptr, &nty);
  }
  // With opts->setup_cached the caller asserts that the workspace and the
  // CSR pattern are untouched since the previous call with this workspace: the
  // count of nonzeros is then not read back, and tables byte-identical to
  // that call's are not copied again (a host->device copy queued behind the
  // caller's own large copies would hold the set-up back).
  SetupCache cache;   // the previous set-up in this workspace (a copy)
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    cache = setup_cache_for(d_work);
  }
  const bool cached = opts && opts->setup_cached && cache.work == d_work &&
                      cache.work_bytes == work_bytes && cache.rowptr == d_rowptr &&
                      cache.col == d_col && cache.B == B && cache.prec == prec_mode &&
                      cache.chunk_rows == chunk_rows &&
                      cache.jacobi == int(needs_jacobi(n_dots, h_prec)) && cache.ntx == ntx &&
                      cache.nty == nty && cache.row_off.size() == size_t(n_dots) + 1 &&
                      std::equal(cache.row_off.begin(), cache.row_off.end(), h_row_off);
  int32_t nnz = 0;   // the CSR's own count of nonzeros
  if (cached) {
    nnz = cache.nnz;
  } else {
    QD_CUDA_TRY(cudaMemcpyAsync(&nnz, d_rowptr + n_rows, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, s));
    QD_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (nnz <= 0) return QD_ERR_INVALID;
  const bool mixed_mode = prec_mode == QD_PREC_MIXED;
  const bool jacobi = needs_jacobi(n_dots, h_prec);
  {
    qd::Arena need(nullptr, 0);
    Layout tmp;
    carve(need, n_dots, n_rows, nnz, B, nchunks, chunk_rows, ntx, nty, mixed_mode, jacobi, tmp);
    if (need.used > work_bytes) return QD_ERR_WORKSPACE;
  }
  if (reinterpret_cast<uintptr_t>(d_work) % 256 != 0) return QD_ERR_WORKSPACE;
  qd::Arena ar(d_work, work_bytes);
  Layout L;
  carve(ar, n_dots, n_rows, nnz, B, nchunks, chunk_rows, ntx, nty, mixed_mode, jacobi, L);
  if (mixed_mode) {
    // FP32 (H, M) pairs scaled by 2^-e, the exponents kept on the device
    hm_exponent_init_kernel<<<1, 32, 0, s>>>(L.hm_exp);
    QD_CHECK_LAUNCH();
    hm_exponent_kernel<<<1184, 256, 0, s>>>(nnz, d_H, d_M, L.hm_exp);
    QD_CHECK_LAUNCH();
    pack_hm32_kernel<<<1184, 256, 0, s>>>(nnz, d_H, d_M, L.hm_exp, L.hm32);
    QD_CHECK_LAUNCH();
    if (!cached)   // the pattern's column indices, with bulk-copy slack
      QD_CUDA_TRY(cudaMemcpyAsync(L.col32, d_col, size_t(nnz) * sizeof(int32_t),
                                  cudaMemcpyDeviceToDevice, s));
    rowsum32_kernel<<<1184, 256, 0, s>>>(n_rows, d_rowptr, L.hm32, L.rs32);
    QD_CHECK_LAUNCH();
  }
  std::vector<qd::GemmTile> htx, hty;
  bool same_tiles = cached;
  if (ntx > 0) {
    if (reinterpret_cast<uintptr_t>(d_mats) % 16) return QD_ERR_INVALID;
    htx.resize(ntx);
    hty.resize(nty);
    qd::dst_tiles(n_dots, h_prec, B, htx.data(), &ntx, hty.data(), &nty, &L.rows_x, &L.rows_y);
    L.mats = d_mats;
    same_tiles = same_tiles && pod_equal(cache.tiles_x, htx) && pod_equal(cache.tiles_y, hty) &&
                 cache.desc.size() == size_t(n_dots) &&
                 std::memcmp(cache.desc.data(), h_prec, n_dots * sizeof(qd_dst_prec)) == 0;
    if (!same_tiles) {
      QD_CUDA_TRY(cudaMemcpyAsync(L.tiles_x, htx.data(), ntx * sizeof(qd::GemmTile),
                                  cudaMemcpyHostToDevice, s));
      QD_CUDA_TRY(cudaMemcpyAsync(L.tiles_y, hty.data(), nty * sizeof(qd::GemmTile),
                                  cudaMemcpyHostToDevice, s));
      QD_CUDA_TRY(cudaMemcpyAsync(L.desc, h_prec, n_dots * sizeof(qd_dst_prec),
                                  cudaMemcpyHostToDevice, s));
    }
  } else {
    same_tiles = same_tiles && cache.tiles_x.empty() && cache.tiles_y.empty();
  }
  // chunk table and per-dot state
  std::vector<Chunk> chunks;
  chunks.reserve(nchunks);
  std::vector<DotState> st(n_dots);
  for (int d = 0; d < n_dots; ++d) {
    DotState &x = st[d];
    std::memset(&x, 0, sizeof(x));
    x.active = 1;
    x.phase = prec_mode == QD_PREC_MIXED ? 0 : 1;
    x.run[x.phase] = 1;
    x.best = 1e300;
    x.chunk0 = int(chunks.size());
    const int jac = (!h_prec || h_prec[d].nx <= 0) ? 1 : 0;
    for (int r = h_row_off[d]; r < h_row_off[d + 1]; r += chunk_rows) {
      chunks.push_back(Chunk{d, r, std::min(r + chunk_rows, h_row_off[d + 1]), jac});
      L.njac += jac;
    }
    x.chunk1 = int(chunks.size());
    if (x.chunk1 == x.chunk0) {
      x.active = 0;
      x.run[0] = x.run[1] = 0;
      x.status = 2;
    }
  }
  const bool same_chunks = cached && same_tiles && pod_equal(cache.chunks, chunks);
  if (!same_chunks) {
    QD_CUDA_TRY(cudaMemcpyAsync(L.chunks, chunks.data(), chunks.size() * sizeof(Chunk),
                                cudaMemcpyHostToDevice, s));
    QD_CUDA_TRY(cudaMemcpyAsync(L.row_off, h_row_off, sizeof(int32_t) * (n_dots + 1),
                                cudaMemcpyHostToDevice, s));
  }
  if (mixed_mode) {
    const int64_t nsubs = int64_t(nchunks) * L.spc, nsubw = int64_t(nchunks) * L.spcw;
    stage_plan_kernel<64><<<int((nsubs + 7) / 8), 256, 0, s>>>(L.chunks, nchunks, L.spc,
                                                               d_rowptr, d_col, L.plan, L.pos16);
    QD_CHECK_LAUNCH();
    stage_plan_kernel<128><<<int((nsubw + 7) / 8), 256, 0, s>>>(
        L.chunks, nchunks, L.spcw, d_rowptr, d_col, L.planw, L.pos16w);
    QD_CHECK_LAUNCH();
  }
  if (L.njac > 0) {
    jacobi_diag_kernel<<<int(chunks.size()), 256, 0, s>>>(L.chunks, d_rowptr, d_col, d_H, L.dinv);
    QD_CHECK_LAUNCH();
  }
  // the per-dot state: from the host, or (same chunk table as the previous
  // call, whose state still holds each dot's chunk range) reset on the device;
  // Theta, the residual norms and the wait flag zeroed by a kernel
  if (!same_chunks)
    QD_CUDA_TRY(cudaMemcpyAsync(L.st, st.data(), st.size() * sizeof(DotState),
                                cudaMemcpyHostToDevice, s));
  state_reset_kernel<<<(n_dots + 127) / 128, 128, 0, s>>>(
      L.st, n_dots, same_chunks ? 1 : 0, prec_mode == QD_PREC_MIXED ? 0 : 1, B, L.theta,
      L.relres, L.wait_err);
  QD_CHECK_LAUNCH();
  // the host tables of this call, for the next call with this workspace
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    SetupCache &c = setup_cache_for(d_work);
    c.work = d_work;
    c.work_bytes = work_bytes;
    c.rowptr = d_rowptr;
    c.col = d_col;
    c.B = B;
    c.prec = prec_mode;
    c.chunk_rows = chunk_rows;
    c.jacobi = jacobi ? 1 : 0;
    c.ntx = ntx;
    c.nty = nty;
    c.nnz = nnz;
    c.row_off.assign(h_row_off, h_row_off + n_dots + 1);
    c.chunks = chunks;
    c.tiles_x = htx;
    c.tiles_y = hty;
    c.desc.clear();
    if (h_prec) c.desc.assign(h_prec, h_prec + n_dots);
  }

  const bool mixed = prec_mode == QD_PREC_MIXED;
  RRParams prm;
  prm.k = k;
  prm.max_iter = max_iter;
  prm.tol = tol;
  prm.tol32 = std::max(100.0 * tol, kTol32Floor);
  prm.stag_window = kStagWindow;
  prm.eig_scale = 0.0;
  prm.mixed = prec_mode == QD_PREC_MIXED ? 1 : 0;
  bool graphs = true;
  const double *x0 = opts ? opts->x0 : nullptr;
  if (opts) {
    if (opts->tol32 > 0.0) prm.tol32 = std::max(opts->tol32, tol);
    if (opts->stag_window > 0) prm.stag_window = opts->stag_window;
    if (opts->eig_scale > 0.0) prm.eig_scale = opts->eig_scale;
    graphs = opts->graphs != 0;
  }
  Bufs<double> b64(L.slot);
  if (mixed) {
    Bufs<float> b32(L.slot32);
    init_kernel<float, B><<<nchunks, 256, 0, s>>>(L.chunks, L.row_off, seed, b32.X, b32.W, b32.P,
                                                  b32.HW, b32.MW, b32.HP, b32.MP, x0, k);
    QD_CHECK_LAUNCH();
  } else {
    init_kernel<double, B><<<nchunks, 256, 0, s>>>(L.chunks, L.row_off, seed, b64.X, b64.W,
                                                   b64.P, b64.HW, b64.MW, b64.HP, b64.MP, x0, k);
    QD_CHECK_LAUNCH();
  }
  int iters_run = 0;
  int rs = run_solver<B>(L, mixed, n_dots, d_rowptr, d_col, d_H, d_M, prm, graphs, s, iters_run);
  if (rs != QD_OK) return rs;
  output_kernel<B><<<nchunks, 256, 0, s>>>(L.chunks, b64.X, k, d_X_out);
  QD_CHECK_LAUNCH();
  finalize_kernel<B><<<(n_dots + 127) / 128, 128, 0, s>>>(L.st, n_dots, k, L.theta, L.relres,
                                                          d_E_out, d_res_out, d_iters_out);
  QD_CHECK_LAUNCH();
  QD_CUDA_TRY(cudaMemcpyAsync(st.data(), L.st, st.size() * sizeof(DotState),
                              cudaMemcpyDeviceToHost, s));
  int wait_err = 0;
  QD_CUDA_TRY(cudaMemcpyAsync(&wait_err, L.wait_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));
  if (wait_err) return QD_ERR_TIMEOUT;
  int nconv = 0, nbreak = 0;
  for (auto &x : st) {
    nconv += (x.status == 1);
    nbreak += (x.status == 2);
  }
  if (h_counts)
    for (int d = 0; d < n_dots; ++d)
      for (int ph = 0; ph < 2; ++ph)
        for (int kd = 0; kd < 3; ++kd) h_counts[d * 6 + ph * 3 + kd] = st[d].launches[ph][kd];
  if (h_info) {
    int it32 = 0, it64 = 0;
    for (auto &x : st) {
      it32 = std::max(it32, x.iters32);
      it64 = std::max(it64, x.iters - x.iters32);
    }
    h_info[0] = iters_run;
    h_info[1] = it32;
    h_info[2] = it64;
    h_info[3] = nconv;
  }
  if (nbreak) return QD_ERR_BREAKDOWN;
  if (nconv != n_dots) return QD_ERR_NOT_CONVERGED;
  return QD_OK;
}

}  // namespace

extern "C" int qd_lobpcg_workspace_size(int32_t n_dots, int64_t n_rows_total,
                                        int64_t nnz_total, int b, int prec_mode,
                                        const qd_dst_prec *h_prec, const qd_lobpcg_opts *opts,
                                        size_t *bytes) {
  if (!bytes || n_dots <= 0 || n_rows_total <= 0 || nnz_total <= 0 || b < 4 || b > kMaxB ||
      b % 4)
    return QD_ERR_INVALID;
  // upper bound on the chunk count: every dot contributes at most one partial chunk
  const int nchunks = int(n_rows_total / chunk_rows_of(opts)) + n_dots;
  int64_t ntx = 0, nty = 0;
  if (h_prec) qd::dst_tiles(n_dots, h_prec, b, nullptr, &ntx, nullptr, &nty);
  qd::Arena ar(nullptr, 0);
  Layout L;
  carve(ar, n_dots, n_rows_total, nnz_total, b, nchunks, chunk_rows_of(opts), ntx, nty,
        prec_mode == QD_PREC_MIXED, needs_jacobi(n_dots, h_prec), L);
  *bytes = ar.used;
  return QD_OK;
}

extern "C" int qd_lobpcg_solve(int32_t n_dots, const int32_t *h_row_off,
                               const int32_t *d_row_off, const int32_t *d_rowptr,
                               const int32_t *d_col, const double *d_H, const double *d_M,
                               const qd_dst_prec *h_prec, const void *d_prec_mats_v, int k,
                               int b, int prec_mode, double tol, int max_iter, uint64_t seed,
                               double *d_X_out, double *d_E_out, double *d_res_out,
                               int32_t *d_iters_out, int32_t *h_info, int32_t *h_counts,
                               void *d_work, size_t work_bytes, const qd_lobpcg_opts *opts,
                               void *stream) {
  (void)d_row_off;
  const uint16_t *d_prec_mats = static_cast<const uint16_t *>(d_prec_mats_v);
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
    case 4: return solve_b<4>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, h_prec, d_prec_mats, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, h_counts, d_work, work_bytes, opts, s);
    case 8: return solve_b<8>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, h_prec, d_prec_mats, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, h_counts, d_work, work_bytes, opts, s);
    case 12: return solve_b<12>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, h_prec, d_prec_mats, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, h_counts, d_work, work_bytes, opts, s);
    default: return solve_b<16>(n_dots, h_row_off, d_rowptr, d_col, d_H, d_M, h_prec, d_prec_mats, k, prec_mode, tol, max_iter, seed, d_X_out, d_E_out, d_res_out, d_iters_out, h_info, h_counts, d_work, work_bytes, opts, s);
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
      qd::spmm_row<TV, B>(r, g, rowptr, col, qd::MatF64{H, M}, X, HX, MX);
    else
      qd::spmv_row<TV, B>(r, g, rowptr, col, H, X, HX);
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

namespace {
// Layout shared by qd_dst_precond_workspace_size and qd_dst_precond_apply.
void carve_precond(qd::Arena &ar, int32_t n_dots, int64_t nv, int64_t ntx, int64_t nty,
                   void **t1, void **t2, qd_dst_prec **desc, int32_t **ro, qd::GemmTile **dtx,
                   qd::GemmTile **dty, int **err) {
  *t1 = ar.take<uint16_t>(size_t(nv));
  *t2 = ar.take<uint16_t>(size_t(nv));
  *desc = ar.take<qd_dst_prec>(n_dots);
  *ro = ar.take<int32_t>(n_dots + 1);
  *dtx = ar.take<qd::GemmTile>(ntx);
  *dty = ar.take<qd::GemmTile>(nty);
  *err = ar.take<int>(1);
}
}  // namespace

extern "C" int qd_dst_matrix_size(int32_t n, int64_t *elems) {
  if (n < 1 || !elems) return QD_ERR_INVALID;
  *elems = qd::tc_mat_elems(n);
  return QD_OK;
}

extern "C" int qd_dst_matrix_fill(int32_t n, uint16_t *h_out) {
  if (n < 1 || !h_out) return QD_ERR_INVALID;
  const int R = qd::tc_rpad(n), KS = qd::tc_ks(n);
  const double scale = std::sqrt(2.0 / double(n + 1));
  auto bf16_bits = [](double x) -> uint16_t {   // round to nearest even via float
    const float f = float(x);
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
  };
  int64_t pos = 0;
  for (int m0 = 0; m0 < R; m0 += qd::kTcRows) {
    const int rows = std::min(qd::kTcRows, R - m0);
    for (int sl = 0; sl < KS; ++sl)
      for (int c = 0; c < 8; ++c)
        for (int g = 0; g < rows / 8; ++g)
          for (int r8 = 0; r8 < 8; ++r8)
            for (int k8 = 0; k8 < 8; ++k8) {
              const int row = m0 + g * 8 + r8, k = sl * qd::kTcK + c * 8 + k8;
              double v = 0.0;
              if (row < n && k < n) {
                // sin(pi (row+1)(k+1)/(n+1)) with the angle reduced exactly in integers
                const int64_t q = (int64_t(row + 1) * (k + 1)) % (2 * int64_t(n + 1));
                v = scale * std::sin(M_PI * double(q) / double(n + 1));
              }
              h_out[pos++] = bf16_bits(v);
            }
  }
  return QD_OK;
}

extern "C" int qd_dst_precond_workspace_size(int32_t n_dots, const int32_t *h_row_off, int b,
                                             const qd_dst_prec *h_prec, size_t *bytes) {
  if (n_dots <= 0 || !h_row_off || !h_prec || !bytes || b < 4) return QD_ERR_INVALID;
  int64_t ntx = 0, nty = 0;
  qd::dst_tiles(n_dots, h_prec, b, nullptr, &ntx, nullptr, &nty);
  qd::Arena ar(nullptr, 0);
  void *t1, *t2;
  qd_dst_prec *desc;
  int32_t *ro;
  qd::GemmTile *dtx, *dty;
  int *err;
  carve_precond(ar, n_dots, int64_t(h_row_off[n_dots]) * b, ntx, nty, &t1, &t2, &desc, &ro,
                &dtx, &dty, &err);
  *bytes = ar.used;
  return QD_OK;
}

extern "C" int qd_dst_precond_apply(int32_t n_dots, const int32_t *h_row_off, int b, int vec_fp32,
                                    const qd_dst_prec *h_prec, const void *d_prec_mats,
                                    const void *d_in, void *d_out, void *d_work,
                                    size_t work_bytes, void *stream) {
  if (n_dots <= 0 || !h_row_off || !h_prec || !d_prec_mats || !d_in || !d_out || !d_work || b < 4)
    return QD_ERR_INVALID;
  if (reinterpret_cast<uintptr_t>(d_prec_mats) % 16) return QD_ERR_INVALID;
  // the transform passes read adjacent column pairs (up to 16 bytes at once)
  if (b % 2 || reinterpret_cast<uintptr_t>(d_in) % 16 || reinterpret_cast<uintptr_t>(d_out) % 16)
    return QD_ERR_INVALID;
  for (int d = 0; d < n_dots; ++d) {
    const qd_dst_prec &q = h_prec[d];
    if (q.nx > 0 && (int64_t(q.nx) * q.ny != h_row_off[d + 1] - h_row_off[d] ||
                     q.sx_off < 0 || q.sy_off < 0 || q.sx_off % 8 || q.sy_off % 8))
      return QD_ERR_INVALID;
  }
  size_t need = 0;
  int st = qd_dst_precond_workspace_size(n_dots, h_row_off, b, h_prec, &need);
  if (st != QD_OK) return st;
  if (need > work_bytes || reinterpret_cast<uintptr_t>(d_work) % 256) return QD_ERR_WORKSPACE;
  int64_t ntx = 0, nty = 0;
  int rows_x = 16, rows_y = 16;
  qd::dst_tiles(n_dots, h_prec, b, nullptr, &ntx, nullptr, &nty);
  std::vector<qd::GemmTile> tx(ntx), ty(nty);
  qd::dst_tiles(n_dots, h_prec, b, tx.data(), &ntx, ty.data(), &nty, &rows_x, &rows_y);
  qd::Arena ar(d_work, work_bytes);
  void *t1, *t2;
  qd_dst_prec *desc;
  int32_t *ro;
  qd::GemmTile *dtx, *dty;
  int *err;
  carve_precond(ar, n_dots, int64_t(h_row_off[n_dots]) * b, ntx, nty, &t1, &t2, &desc, &ro,
                &dtx, &dty, &err);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  QD_CUDA_TRY(cudaMemcpyAsync(desc, h_prec, n_dots * sizeof(qd_dst_prec), cudaMemcpyHostToDevice, s));
  QD_CUDA_TRY(cudaMemcpyAsync(ro, h_row_off, (n_dots + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (ntx) QD_CUDA_TRY(cudaMemcpyAsync(dtx, tx.data(), ntx * sizeof(qd::GemmTile), cudaMemcpyHostToDevice, s));
  if (nty) QD_CUDA_TRY(cudaMemcpyAsync(dty, ty.data(), nty * sizeof(qd::GemmTile), cudaMemcpyHostToDevice, s));
  QD_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
  const uint16_t *mats = static_cast<const uint16_t *>(d_prec_mats);
  cudaError_t e;
  if (vec_fp32)
    e = qd::dst_apply<float>(dtx, ntx, rows_x, dty, nty, rows_y, nullptr, 0, desc, ro, mats, b,
                             static_cast<const float *>(d_in), static_cast<float *>(d_out), t1,
                             t2, err, s);
  else
    e = qd::dst_apply<double>(dtx, ntx, rows_x, dty, nty, rows_y, nullptr, 0, desc, ro, mats, b,
                              static_cast<const double *>(d_in), static_cast<double *>(d_out),
                              t1, t2, err, s);
  if (e != cudaSuccess) return QD_ERR_CUDA;
  int herr = 0;
  QD_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  QD_CUDA_TRY(cudaStreamSynchronize(s));   // host tile tables die at return
  return herr ? QD_ERR_TIMEOUT : QD_OK;
}
