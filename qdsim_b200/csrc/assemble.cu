// Warp-per-row finite-element assembly into a precomputed CSR pattern.
//
// Replaces FEMSolver::assemble_element_matrix (backend/src/fem.cpp:736-990),
// the per-element / batched GPU element kernels (backend/src/gpu_kernels.cu:
// 46-336, 442-745) and the host triplet scatter of
// GPUAccelerator::assemble_matrices (backend/src/gpu_accelerator.cpp:439-642).
//
// Each reduced row r is owned by a segment of 8 (P1), 16 (P2) or 32 (P3)
// lanes, so a warp advances 4, 2 or 1 rows at once.  The segment first stages
// the row's incident elements (geometry, coefficient, nodal V/W) in shared
// memory, then each lane owns CSR slots of the row and sums each slot's
// contributions in the fixed (element id, local column) order given by the
// host plan.  No atomics, so the
// result is bitwise reproducible; every slot is written exactly once and the
// row's slots are contiguous, so stores are coalesced.
//
// Element formulas (per element, A = area, Ginv = J^-1 J^-T):
//   FEM:        H_ab = c A (g00 Sxx + g01 Sxy + g11 Syy)_ab + A sum_l V_l T_lab
//               M_ab = A Mr_ab,  Himag_ab = -A sum_l W_l T_lab
//   REF_CYTHON: schrodinger_solver.pyx:201-251 -- correct P1 stiffness, element
//               V lumped as V A/3 on the diagonal, added a second time at local
//               nodes 1 and 2 (:224-236); consistent mass.
//   REF_FIXED:  fixed_open_system_solver.pyx:225-255 -- c A/3 on the diagonal and
//               c A/6 off it (no gradients), V A/3 on the diagonal; consistent mass.
//   REF_CPP:    SchrodingerSolver::assemble_matrices_cpu (backend/src/schrodinger.cpp:
//               92-230) -- correct P1 stiffness; the potential and the mass by the
//               one-point centroid rule, every entry V A/9 and A/9.
#include <cuda_runtime.h>
#include "common.h"
#include "devtables.cuh"

namespace qd {
std::atomic<uint64_t> g_launches{0};
}

namespace {

constexpr int kMaxAdj = 16;   // incident elements per row (pattern builder enforces)

// Lanes per row and threads per block by element order: a P1 row has at most
// 7 slots in a structured mesh, a P2 row 19, a P3 row 37, so P1 rows get 8
// lanes (four rows per warp), P2 rows 16 (two per warp), P3 rows a warp.
template <int K> struct RowShape;
template <> struct RowShape<3> { static constexpr int LPR = 8, THREADS = 128; };
template <> struct RowShape<6> { static constexpr int LPR = 16, THREADS = 128; };
template <> struct RowShape<10> { static constexpr int LPR = 32, THREADS = 128; };

// One row's staged data: the incident elements' geometry and nodal V (W),
// then the row's element-matrix entries (t, b) = row a_t of element t's H, M
// (and Himag) at local column b, each computed once by one lane.
template <int K, bool HAS_W>
struct __align__(16) RowStage {
  double cA[kMaxAdj], A[kMaxAdj], g00[kMaxAdj], g01[kMaxAdj], g11[kMaxAdj];
  double V[kMaxAdj][K];
  double W[HAS_W ? kMaxAdj : 1][K];
  double he[kMaxAdj][K], me[kMaxAdj][K];
  double we[HAS_W ? kMaxAdj : 1][K];
  int a[kMaxAdj];
};

// HAS_W: a CAP amplitude is given (Himag is assembled); without it the W
// staging and the W sums are compiled out.
template <int K, bool HAS_W>
__global__ void __launch_bounds__(RowShape<K>::THREADS)
assemble_rows_kernel(int mode, int32_t n, const double2 *__restrict__ nodes,
                     const int32_t *__restrict__ elems, const double *__restrict__ cvec,
                     const double *__restrict__ V, const double *__restrict__ W,
                     const int32_t *__restrict__ rowptr, const int32_t *__restrict__ adjptr,
                     const int32_t *__restrict__ adj, const int32_t *__restrict__ cptr,
                     const uint8_t *__restrict__ contrib, const uint8_t *__restrict__ slotcnt,
                     double *__restrict__ H, double *__restrict__ M, double *__restrict__ Him,
                     int32_t *__restrict__ status) {
  constexpr int KK = K * K;
  constexpr int NT = 4 * KK + K * KK;
  constexpr int LPR = RowShape<K>::LPR;
  constexpr int RPB = RowShape<K>::THREADS / LPR;   // rows in flight per block
  __shared__ __align__(16) double s_tab[NT];
  __shared__ RowStage<K, HAS_W> s_stage[RPB];
  // Mr, Sxx, Sxy, Syy as stored; the potential table transposed to T[ab][l]
  // so that a contribution reads its K weights contiguously
  for (int i = threadIdx.x; i < NT; i += blockDim.x) {
    if (i < 4 * KK) {
      s_tab[i] = c_tab[TabBase<K>::v + i];
    } else {
      const int l = (i - 4 * KK) / KK, ab = (i - 4 * KK) % KK;
      s_tab[4 * KK + ab * K + l] = c_tab[TabBase<K>::v + i];
    }
  }
  __syncthreads();
  const double *Mr = s_tab, *Sxx = s_tab + KK, *Sxy = s_tab + 2 * KK, *Syy = s_tab + 3 * KK;
  const double *T = s_tab + 4 * KK;
  const int seg = threadIdx.x / LPR, lane = threadIdx.x % LPR;
  RowStage<K, HAS_W> &st = s_stage[seg];
  // rows of one warp are independent: every shuffle and warp barrier names
  // only the lanes of this row's segment
  const unsigned mask = LPR == 32 ? 0xffffffffu
                                  : ((1u << (LPR & 31)) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1));

  for (int32_t r = blockIdx.x * RPB + seg; r < n; r += gridDim.x * RPB) {
    const int t0 = adjptr[r];
    const int m = adjptr[r + 1] - t0;
    for (int t = lane; t < m; t += LPR) {
      const int packed = adj[t0 + t];
      const int e = packed >> 4;
      const double2 p0 = nodes[elems[e * K + 0]];
      const double2 p1 = nodes[elems[e * K + 1]];
      const double2 p2 = nodes[elems[e * K + 2]];
      const double ja = p1.x - p0.x, jb = p2.x - p0.x, jc = p1.y - p0.y, jd = p2.y - p0.y;
      const double det = ja * jd - jb * jc;
      const double A = 0.5 * fabs(det);
      const double inv2 = 1.0 / (det * det);
      const double ce = cvec[e];
      st.g00[t] = (jd * jd + jb * jb) * inv2;
      st.g01[t] = -(jd * jc + jb * ja) * inv2;
      st.g11[t] = (jc * jc + ja * ja) * inv2;
      st.cA[t] = ce * A;
      st.A[t] = A;
      st.a[t] = packed & 15;
      if (!(det != 0.0) || !isfinite(det) || !isfinite(ce)) atomicOr(status, 1);
      if (mode != QD_ASM_FEM) {
        const double ve = V[e];
        st.V[t][0] = ve;
        if (!isfinite(ve)) atomicOr(status, 2);
      }
    }
    if (mode == QD_ASM_FEM) {
      for (int idx = lane; idx < m * K; idx += LPR) {
        const int t = idx / K, l = idx - t * K;
        const int e = adj[t0 + t] >> 4;
        const int g = elems[e * K + l];
        const double v = V[g];
        st.V[t][l] = v;
        if (HAS_W) st.W[t][l] = W[g];
        if (!isfinite(v)) atomicOr(status, 2);
      }
    }
    __syncwarp(mask);
    // the row's element-matrix entries: lane per (element t, local column b)
    for (int idx = lane; idx < m * K; idx += LPR) {
      const int t = idx / K, b = idx - t * K;
      const int a = st.a[t];
      const int ab = a * K + b;
      const double At = st.A[t];
      double hk, mk, wk = 0.0;
      if (mode == QD_ASM_FEM) {
        hk = st.cA[t] * (st.g00[t] * Sxx[ab] + st.g01[t] * Sxy[ab] + st.g11[t] * Syy[ab]);
        const double *tw = T + ab * K;
        double vs = 0.0, ws = 0.0;
        if constexpr (K % 2 == 0) {
          const double2 *t2 = reinterpret_cast<const double2 *>(tw);
          const double2 *v2 = reinterpret_cast<const double2 *>(st.V[t]);
#pragma unroll
          for (int l = 0; l < K / 2; ++l) {
            const double2 tl = t2[l], vl = v2[l];
            vs += vl.x * tl.x;
            vs += vl.y * tl.y;
          }
          if constexpr (HAS_W) {
            const double2 *w2 = reinterpret_cast<const double2 *>(st.W[t]);
#pragma unroll
            for (int l = 0; l < K / 2; ++l) {
              const double2 tl = t2[l], wl = w2[l];
              ws += wl.x * tl.x;
              ws += wl.y * tl.y;
            }
          }
        } else {
#pragma unroll
          for (int l = 0; l < K; ++l) {
            vs += st.V[t][l] * tw[l];
            if constexpr (HAS_W) ws += st.W[t][l] * tw[l];
          }
        }
        hk += At * vs;
        wk = At * ws;
        mk = At * Mr[ab];
      } else if (mode == QD_ASM_REF_CYTHON) {
        hk = st.cA[t] * (st.g00[t] * Sxx[ab] + st.g01[t] * Sxy[ab] + st.g11[t] * Syy[ab]);
        if (a == b) hk += (a == 0 ? 1.0 : 2.0) * (st.V[t][0] * At / 3.0);
        mk = At * Mr[ab];
      } else if (mode == QD_ASM_REF_FIXED) {
        hk = (st.cA[t] / 3.0) * (a == b ? 1.0 : 0.5);
        if (a == b) hk += st.V[t][0] * At / 3.0;
        mk = At * Mr[ab];
      } else {
        hk = st.cA[t] * (st.g00[t] * Sxx[ab] + st.g01[t] * Sxy[ab] + st.g11[t] * Syy[ab]) +
             st.V[t][0] * At / 9.0;
        mk = At / 9.0;
      }
      st.he[t][b] = hk;
      st.me[t][b] = mk;
      if constexpr (HAS_W) st.we[t][b] = wk;
    }
    __syncwarp(mask);
    const int rp = rowptr[r];
    const int L = rowptr[r + 1] - rp;
    const int cbase = cptr[r];
    int carry = 0;
    for (int s0 = 0; s0 < L; s0 += LPR) {
      const int s = s0 + lane;
      const int cnt = (s < L) ? int(slotcnt[rp + s]) : 0;
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < LPR; o <<= 1) {
        const int y = __shfl_up_sync(mask, incl, o, LPR);
        if (lane >= o) incl += y;
      }
      const int start = carry + incl - cnt;
      carry += __shfl_sync(mask, incl, LPR - 1, LPR);
      if (s < L) {
        // the slot's contributions in the plan's order (bitwise reproducible)
        double h = 0.0, mm = 0.0, wi = 0.0;
        for (int q = 0; q < cnt; ++q) {
          const int id = contrib[cbase + start + q];
          const int t = id / K, b = id - t * K;
          h += st.he[t][b];
          mm += st.me[t][b];
          if constexpr (HAS_W) wi -= st.we[t][b];
        }
        H[rp + s] = h;
        M[rp + s] = mm;
        if (Him) Him[rp + s] = wi;
      }
    }
    __syncwarp(mask);
  }
}

template <int K>
int launch_assemble(int mode, int32_t n, const double *nodes, const int32_t *elems,
                    const double *c, const double *V, const double *W, const int32_t *rowptr,
                    const int32_t *adjptr, const int32_t *adj, const int32_t *cptr,
                    const uint8_t *contrib, const uint8_t *slotcnt, double *H, double *M,
                    double *Him, int32_t *status, cudaStream_t s) {
  if (n == 0) return QD_OK;
  constexpr int RPB = RowShape<K>::THREADS / RowShape<K>::LPR;
  int64_t blocks = (int64_t(n) + RPB - 1) / RPB;
  if (blocks > 148 * 64) blocks = 148 * 64;
  qd::prof_begin(qd::PK_ASSEMBLE, s);
  if (W && mode == QD_ASM_FEM)
    assemble_rows_kernel<K, true><<<int(blocks), RowShape<K>::THREADS, 0, s>>>(
        mode, n, reinterpret_cast<const double2 *>(nodes), elems, c, V, W, rowptr, adjptr, adj,
        cptr, contrib, slotcnt, H, M, Him, status);
  else
    assemble_rows_kernel<K, false><<<int(blocks), RowShape<K>::THREADS, 0, s>>>(
        mode, n, reinterpret_cast<const double2 *>(nodes), elems, c, V, W, rowptr, adjptr, adj,
        cptr, contrib, slotcnt, H, M, Him, status);
  qd::prof_end(qd::PK_ASSEMBLE, s);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

}  // namespace

extern "C" int qd_assemble(int order, int mode, int64_t num_nodes, int64_t num_elems,
                           int32_t n_dofs, const double *d_nodes, const int32_t *d_elems,
                           const double *d_c, const double *d_V, const double *d_W,
                           const int32_t *d_rowptr, const int32_t *d_adjptr,
                           const int32_t *d_adj, const int32_t *d_cptr,
                           const uint8_t *d_contrib, const uint8_t *d_slotcnt, double *d_H,
                           double *d_M, double *d_Himag, int32_t *d_status, void *stream) {
  if (order < 1 || order > 3) return QD_ERR_INVALID;
  if (mode != QD_ASM_FEM && mode != QD_ASM_REF_CYTHON && mode != QD_ASM_REF_FIXED &&
      mode != QD_ASM_REF_CPP)
    return QD_ERR_INVALID;
  if (mode != QD_ASM_FEM && order != 1) return QD_ERR_INVALID;
  if (num_nodes <= 0 || num_elems <= 0 || n_dofs < 0) return QD_ERR_INVALID;
  if (!d_nodes || !d_elems || !d_c || !d_V || !d_rowptr || !d_adjptr || !d_adj || !d_cptr ||
      !d_contrib || !d_slotcnt || !d_H || !d_M || !d_status)
    return QD_ERR_INVALID;
  if (reinterpret_cast<uintptr_t>(d_nodes) % 16 != 0) return QD_ERR_INVALID;
  int st = ensure_tables();
  if (st != QD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (order) {
    case 1:
      return launch_assemble<3>(mode, n_dofs, d_nodes, d_elems, d_c, d_V, d_W, d_rowptr,
                                d_adjptr, d_adj, d_cptr, d_contrib, d_slotcnt, d_H, d_M,
                                d_Himag, d_status, s);
    case 2:
      return launch_assemble<6>(mode, n_dofs, d_nodes, d_elems, d_c, d_V, d_W, d_rowptr,
                                d_adjptr, d_adj, d_cptr, d_contrib, d_slotcnt, d_H, d_M,
                                d_Himag, d_status, s);
    default:
      return launch_assemble<10>(mode, n_dofs, d_nodes, d_elems, d_c, d_V, d_W, d_rowptr,
                                 d_adjptr, d_adj, d_cptr, d_contrib, d_slotcnt, d_H, d_M,
                                 d_Himag, d_status, s);
  }
}

extern "C" const char *qd_version(void) { return "qdsim_b200 0.1.0 (sm_100a)"; }

extern "C" uint64_t qd_kernel_launch_count(void) {
  return qd::g_launches.load(std::memory_order_relaxed);
}

extern "C" const char *qd_status_string(int status) {
  switch (status) {
    case QD_OK: return "ok";
    case QD_ERR_INVALID: return "invalid argument";
    case QD_ERR_CUDA: return "CUDA runtime error";
    case QD_ERR_NOT_CONVERGED: return "not converged";
    case QD_ERR_BREAKDOWN: return "breakdown (Gram matrix not positive definite)";
    case QD_ERR_WORKSPACE: return "workspace too small";
    case QD_ERR_DEGENERATE: return "degenerate element or non-finite coefficient";
    case QD_ERR_LIMIT: return "size exceeds a compiled-in limit";
    case QD_ERR_TIMEOUT: return "device-side wait exceeded its time bound";
    default: return "unknown status";
  }
}
