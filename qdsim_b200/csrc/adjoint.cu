// Adjoint (Hellmann-Feynman) gradients of L = sum_s w_s E_s.
//
// With M-normalised eigenvectors and M independent of V and c,
//   dE_s/dV_g = psi_s^T (dH/dV_g) psi_s = sum_{e ∋ g, local l} A_e sum_ij T_lij psi_i psi_j
//   dE_s/dc_e = psi_s^T Khat_e psi_s,   Khat_e = A_e (g00 Sxx + g01 Sxy + g11 Syy)
// (same element formulas as the assembly kernel).  The nodal gradient is a
// gather over each node's incident elements in a fixed order, so the result is
// reproducible without atomics.  The reference has no derivatives; the checks
// are central finite differences of FP64 eigenvalues and an FP64 oracle.
#include <cuda_runtime.h>
#include <algorithm>
#include "common.h"
#include "devtables.cuh"

namespace {

constexpr int kMaxStates = 16;

template <int K>
__device__ inline void element_geom(int e, const double2 *nodes, const int32_t *elems, double &A,
                                    double &g00, double &g01, double &g11) {
  const double2 p0 = nodes[elems[e * K + 0]];
  const double2 p1 = nodes[elems[e * K + 1]];
  const double2 p2 = nodes[elems[e * K + 2]];
  const double ja = p1.x - p0.x, jb = p2.x - p0.x, jc = p1.y - p0.y, jd = p2.y - p0.y;
  const double det = ja * jd - jb * jc;
  A = 0.5 * fabs(det);
  const double inv2 = 1.0 / (det * det);
  g00 = (jd * jd + jb * jb) * inv2;
  g01 = -(jd * jc + jb * ja) * inv2;
  g11 = (jc * jc + ja * ja) * inv2;
}

// U_ij = sum_s w_s psi_s(i) psi_s(j) for the element's local nodes
template <int K>
__device__ inline void element_u(int e, int ns, const int32_t *elems, const int32_t *dofmap,
                                 const double *psi, const double *w, double (&u)[K][K]) {
  double v[K][kMaxStates];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const int dof = dofmap[elems[e * K + i]];
    for (int s = 0; s < ns; ++s) v[i][s] = dof >= 0 ? psi[size_t(dof) * ns + s] : 0.0;
  }
#pragma unroll
  for (int i = 0; i < K; ++i)
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double acc = 0.0;
      for (int s = 0; s < ns; ++s) acc = fma(w[s] * v[i][s], v[j][s], acc);
      u[i][j] = acc;
    }
}

template <int K>
__global__ void adjoint_c_kernel(int64_t ne, int ns, const double2 *nodes, const int32_t *elems,
                                 const int32_t *dofmap, const double *psi, const double *w,
                                 double *dLdc) {
  constexpr int KK = K * K;
  __shared__ double s_tab[3 * KK];
  for (int i = threadIdx.x; i < 3 * KK; i += blockDim.x)
    s_tab[i] = c_tab[TabBase<K>::v + KK + i];   // Sxx, Sxy, Syy
  __syncthreads();
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < ne;
       e += int64_t(gridDim.x) * blockDim.x) {
    double A, g00, g01, g11;
    element_geom<K>(int(e), nodes, elems, A, g00, g01, g11);
    double u[K][K];
    element_u<K>(int(e), ns, elems, dofmap, psi, w, u);
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const int ij = i * K + j;
        acc += (g00 * s_tab[ij] + g01 * s_tab[KK + ij] + g11 * s_tab[2 * KK + ij]) * u[i][j];
      }
    dLdc[e] = A * acc;
  }
}

template <int K>
__global__ void adjoint_v_kernel(int64_t nn, int ns, const double2 *nodes, const int32_t *elems,
                                 const int32_t *dofmap, const double *psi, const double *w,
                                 const int32_t *nadjptr, const int32_t *nadj, double *dLdV) {
  constexpr int KK = K * K;
  __shared__ double s_T[K * KK];
  for (int i = threadIdx.x; i < K * KK; i += blockDim.x)
    s_T[i] = c_tab[TabBase<K>::v + 4 * KK + i];
  __syncthreads();
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < nn;
       g += int64_t(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (int t = nadjptr[g]; t < nadjptr[g + 1]; ++t) {
      const int packed = nadj[t];
      const int e = packed >> 4, l = packed & 15;
      double A, g00, g01, g11;
      element_geom<K>(e, nodes, elems, A, g00, g01, g11);
      double u[K][K];
      element_u<K>(e, ns, elems, dofmap, psi, w, u);
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < K; ++i)
#pragma unroll
        for (int j = 0; j < K; ++j) s = fma(s_T[l * KK + i * K + j], u[i][j], s);
      acc += A * s;
    }
    dLdV[g] = acc;
  }
}

template <int K>
int launch_adjoint(int64_t nn, int64_t ne, int ns, const double *nodes, const int32_t *elems,
                   const int32_t *dofmap, const double *psi, const double *w,
                   const int32_t *nadjptr, const int32_t *nadj, double *dLdV, double *dLdc,
                   cudaStream_t s) {
  const double2 *nd = reinterpret_cast<const double2 *>(nodes);
  int bc = int(std::min<int64_t>((ne + 127) / 128, 148 * 16));
  adjoint_c_kernel<K><<<bc, 128, 0, s>>>(ne, ns, nd, elems, dofmap, psi, w, dLdc);
  QD_CHECK_LAUNCH();
  int bv = int(std::min<int64_t>((nn + 127) / 128, 148 * 16));
  adjoint_v_kernel<K><<<bv, 128, 0, s>>>(nn, ns, nd, elems, dofmap, psi, w, nadjptr, nadj, dLdV);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

}  // namespace

extern "C" int qd_adjoint(int order, int64_t num_nodes, int64_t num_elems, int n_states,
                          const double *d_nodes, const int32_t *d_elems, const int32_t *d_dofmap,
                          const double *d_c, const double *d_psi, const double *d_w,
                          const int32_t *d_nadjptr, const int32_t *d_nadj, double *d_dLdV,
                          double *d_dLdc, void *stream) {
  (void)d_c;
  if (order < 1 || order > 3 || num_nodes <= 0 || num_elems <= 0) return QD_ERR_INVALID;
  if (n_states < 1 || n_states > kMaxStates) return QD_ERR_LIMIT;
  if (!d_nodes || !d_elems || !d_dofmap || !d_psi || !d_w || !d_nadjptr || !d_nadj || !d_dLdV ||
      !d_dLdc)
    return QD_ERR_INVALID;
  int st = ensure_tables();
  if (st != QD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (order) {
    case 1: return launch_adjoint<3>(num_nodes, num_elems, n_states, d_nodes, d_elems, d_dofmap, d_psi, d_w, d_nadjptr, d_nadj, d_dLdV, d_dLdc, s);
    case 2: return launch_adjoint<6>(num_nodes, num_elems, n_states, d_nodes, d_elems, d_dofmap, d_psi, d_w, d_nadjptr, d_nadj, d_dLdV, d_dLdc, s);
    default: return launch_adjoint<10>(num_nodes, num_elems, n_states, d_nodes, d_elems, d_dofmap, d_psi, d_w, d_nadjptr, d_nadj, d_dLdV, d_dLdc, s);
  }
}
