// Adjoint (Hellmann-Feynman) gradients of L = Re sum_s w_s E_s.
//
// For the Hermitian pencil (H, M) with M-normalised real eigenvectors and for
// the complex-symmetric open-system pencil (H + i Himag, M) with bilinearly
// normalised complex eigenvectors (x^T M x = 1, no conjugation, so that the
// left eigenvector is x itself), M depends on neither V nor c and
//   dE_s/dp = x_s^T (dH/dp) x_s.
// Per element e with local nodes i, j and U_ij = Re sum_s w_s x_si x_sj
// (complex weights w_s = dL/dRe E_s - i dL/dIm E_s):
//   dL/dV_g = sum_{(e, l): node g} A_e sum_ij T_lij U_ij
//   dL/dc_e = A_e sum_ij (g00 Sxx + g01 Sxy + g11 Syy)_ij U_ij
// with the assembly kernel's reference tables (T_lij = int phi_l phi_i phi_j
// on the reference triangle).
//
// Two launches.  The element pass gives each element to a group of GS lanes
// (8 / 16 / 32 for P1 / P2 / P3, persistent blocks): the group stages the
// element's K x n_states amplitudes in shared memory, each lane owns a few of
// the K^2 (i, j) pairs and forms U_ij and its contributions, and the group
// sums by shuffles into dL/dc_e and the element's K nodal contributions
// (caller scratch, num_elems x K).  The node pass sums each node's
// contributions over its incident elements in adjacency order, so every
// result is reproducible without atomics, and each element is evaluated once.  No reference counterpart (the reference has no derivatives);
// checked against central finite differences and the FP64 oracle gradient.
#include <cuda_runtime.h>
#include <algorithm>
#include "common.h"
#include "devtables.cuh"

namespace {

constexpr int kMaxStates = 16;
constexpr int kThreads = 256;

template <int K> struct AdjCfg;
template <> struct AdjCfg<3> { static constexpr int GS = 8; };
template <> struct AdjCfg<6> { static constexpr int GS = 16; };
template <> struct AdjCfg<10> { static constexpr int GS = 32; };

template <int K>
__device__ inline void element_geom(int e, const double2 *nodes, const int32_t *elems, double &A,
                                    double &g00, double &g01, double &g11) {
  const double2 p0 = nodes[elems[size_t(e) * K + 0]];
  const double2 p1 = nodes[elems[size_t(e) * K + 1]];
  const double2 p2 = nodes[elems[size_t(e) * K + 2]];
  const double ja = p1.x - p0.x, jb = p2.x - p0.x, jc = p1.y - p0.y, jd = p2.y - p0.y;
  const double det = ja * jd - jb * jc;
  A = 0.5 * fabs(det);
  const double inv2 = 1.0 / (det * det);
  g00 = (jd * jd + jb * jb) * inv2;
  g01 = -(jd * jc + jb * ja) * inv2;
  g11 = (jc * jc + ja * ja) * inv2;
}

// Sum over the GS lanes of a group (mask: the group's lanes; groups of one
// warp may be on different units, so the shuffles name only their own lanes).
template <int GS>
__device__ inline double group_sum(double v, unsigned mask) {
#pragma unroll
  for (int o = GS / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, GS);
  return v;
}

// Stage the amplitudes of element e (K nodes x ns states, real and, for a
// complex pencil, imaginary parts) in the group's shared slice.
template <int K, int GS, bool CPLX>
__device__ inline void stage_element(int e, int ns, int lane, const int32_t *elems,
                                     const int32_t *dofmap, const double *psi, double *s_re,
                                     double *s_im, unsigned mask) {
  for (int idx = lane; idx < K * ns; idx += GS) {
    const int i = idx / ns, s = idx - i * ns;
    const int dof = dofmap[elems[size_t(e) * K + i]];
    double re = 0.0, im = 0.0;
    if (dof >= 0) {
      if (CPLX) {
        const double2 z = reinterpret_cast<const double2 *>(psi)[size_t(dof) * ns + s];
        re = z.x;
        im = z.y;
      } else {
        re = psi[size_t(dof) * ns + s];
      }
    }
    s_re[i * ns + s] = re;
    if (CPLX) s_im[i * ns + s] = im;
  }
  __syncwarp(mask);
}

// U_ij = Re sum_s w_s x_si x_sj for the pair (i, j)
template <bool CPLX>
__device__ inline double pair_u(int i, int j, int ns, const double *s_re, const double *s_im,
                                const double *s_w) {
  double u = 0.0;
  for (int s = 0; s < ns; ++s) {
    const double ri = s_re[i * ns + s], rj = s_re[j * ns + s];
    if (CPLX) {
      const double ii = s_im[i * ns + s], ij = s_im[j * ns + s];
      const double pr = ri * rj - ii * ij, pi = ri * ij + ii * rj;
      u = fma(s_w[2 * s], pr, fma(-s_w[2 * s + 1], pi, u));
    } else {
      u = fma(s_w[s] * ri, rj, u);
    }
  }
  return u;
}

// Pass 1, one element per group: dL/dc_e and the element's contribution to
// each of its K nodes' dL/dV, gl[e][l] = A_e sum_ij T_lij U_ij.
template <int K, bool CPLX>
__global__ void __launch_bounds__(kThreads)
adjoint_elem_kernel(int64_t ne, int ns, const double2 *__restrict__ nodes,
                    const int32_t *__restrict__ elems, const int32_t *__restrict__ dofmap,
                    const double *__restrict__ psi, const double *__restrict__ w,
                    double *__restrict__ dLdc, double *__restrict__ gl) {
  constexpr int KK = K * K;
  constexpr int GS = AdjCfg<K>::GS;
  constexpr int NG = kThreads / GS;
  constexpr int PP = (KK + GS - 1) / GS;        // pairs per lane
  __shared__ double s_S[3 * KK];                // Sxx, Sxy, Syy
  __shared__ double s_T[K * KK];                // T[l][i][j]
  __shared__ double s_w[2 * kMaxStates];
  __shared__ double s_amp[NG][2 * K * kMaxStates];
  for (int i = threadIdx.x; i < 3 * KK; i += blockDim.x) s_S[i] = c_tab[TabBase<K>::v + KK + i];
  for (int i = threadIdx.x; i < K * KK; i += blockDim.x)
    s_T[i] = c_tab[TabBase<K>::v + 4 * KK + i];
  if (threadIdx.x < (CPLX ? 2 : 1) * ns) s_w[threadIdx.x] = w[threadIdx.x];
  __syncthreads();

  const int grp = threadIdx.x / GS, lane = threadIdx.x % GS;
  const unsigned mask =
      GS == 32 ? 0xffffffffu : (((1u << GS) - 1u) << ((threadIdx.x & 31) / GS * GS));
  double *s_re = s_amp[grp];
  double *s_im = s_re + K * ns;
  for (int64_t u = int64_t(blockIdx.x) * NG + grp; u < ne; u += int64_t(gridDim.x) * NG) {
    const int e = int(u);
    double A, g00, g01, g11;
    element_geom<K>(e, nodes, elems, A, g00, g01, g11);
    stage_element<K, GS, CPLX>(e, ns, lane, elems, dofmap, psi, s_re, s_im, mask);
    double acc_c = 0.0, acc[K];
#pragma unroll
    for (int l = 0; l < K; ++l) acc[l] = 0.0;
#pragma unroll
    for (int q = 0; q < PP; ++q) {
      const int ij = lane + q * GS;
      if (ij < KK) {
        const int i = ij / K, j = ij - i * K;
        const double uij = pair_u<CPLX>(i, j, ns, s_re, s_im, s_w);
        const double kh = g00 * s_S[ij] + g01 * s_S[KK + ij] + g11 * s_S[2 * KK + ij];
        acc_c = fma(kh, uij, acc_c);
#pragma unroll
        for (int l = 0; l < K; ++l) acc[l] = fma(s_T[l * KK + ij], uij, acc[l]);
      }
    }
    acc_c = group_sum<GS>(acc_c, mask);
#pragma unroll
    for (int l = 0; l < K; ++l) acc[l] = group_sum<GS>(acc[l], mask);
    if (lane == 0) dLdc[e] = A * acc_c;
    if (lane < K) {
      double v = 0.0;
#pragma unroll
      for (int l = 0; l < K; ++l) v = (lane == l) ? acc[l] : v;
      gl[size_t(e) * K + lane] = A * v;
    }
    __syncwarp(mask);
  }
}

// Pass 2, one thread per node: dL/dV_g = sum over the node's incident
// (element, local index) pairs, in adjacency order, of gl[e][l].
template <int K>
__global__ void adjoint_node_kernel(int64_t nn, const int32_t *__restrict__ nadjptr,
                                    const int32_t *__restrict__ nadj,
                                    const double *__restrict__ gl, double *__restrict__ dLdV) {
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < nn;
       g += int64_t(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (int t = nadjptr[g]; t < nadjptr[g + 1]; ++t) {
      const int packed = nadj[t];
      acc += gl[size_t(packed >> 4) * K + (packed & 15)];
    }
    dLdV[g] = acc;
  }
}

template <int K>
int launch_adjoint(int64_t nn, int64_t ne, int ns, bool cplx, const double *nodes,
                   const int32_t *elems, const int32_t *dofmap, const double *psi,
                   const double *w, const int32_t *nadjptr, const int32_t *nadj, double *dLdV,
                   double *dLdc, double *gl, cudaStream_t s) {
  const double2 *nd = reinterpret_cast<const double2 *>(nodes);
  constexpr int NG = kThreads / AdjCfg<K>::GS;
  const int eblocks = int(std::min<int64_t>((ne + NG - 1) / NG, 148 * 8));
  qd::prof_begin(qd::PK_ADJOINT, s);
  if (cplx)
    adjoint_elem_kernel<K, true><<<eblocks, kThreads, 0, s>>>(ne, ns, nd, elems, dofmap, psi, w,
                                                             dLdc, gl);
  else
    adjoint_elem_kernel<K, false><<<eblocks, kThreads, 0, s>>>(ne, ns, nd, elems, dofmap, psi,
                                                              w, dLdc, gl);
  QD_CHECK_LAUNCH();
  const int nblocks = int(std::min<int64_t>((nn + 255) / 256, 148 * 16));
  adjoint_node_kernel<K><<<nblocks, 256, 0, s>>>(nn, nadjptr, nadj, gl, dLdV);
  QD_CHECK_LAUNCH();
  qd::prof_end(qd::PK_ADJOINT, s);
  return QD_OK;
}

}  // namespace

extern "C" int qd_adjoint(int order, int64_t num_nodes, int64_t num_elems, int n_states,
                          int is_complex, const double *d_nodes, const int32_t *d_elems,
                          const int32_t *d_dofmap, const double *d_psi, const double *d_w,
                          const int32_t *d_nadjptr, const int32_t *d_nadj, double *d_dLdV,
                          double *d_dLdc, double *d_work, void *stream) {
  if (order < 1 || order > 3 || num_nodes <= 0 || num_elems <= 0) return QD_ERR_INVALID;
  if (n_states < 1 || n_states > kMaxStates) return QD_ERR_LIMIT;
  if (num_elems >= (int64_t(1) << 27) || num_nodes >= (int64_t(1) << 31)) return QD_ERR_LIMIT;
  if (!d_nodes || !d_elems || !d_dofmap || !d_psi || !d_w || !d_nadjptr || !d_nadj || !d_dLdV ||
      !d_dLdc || !d_work)
    return QD_ERR_INVALID;
  if (is_complex && (reinterpret_cast<uintptr_t>(d_psi) & 15)) return QD_ERR_INVALID;
  int st = ensure_tables();
  if (st != QD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool c = is_complex != 0;
  switch (order) {
    case 1: return launch_adjoint<3>(num_nodes, num_elems, n_states, c, d_nodes, d_elems, d_dofmap, d_psi, d_w, d_nadjptr, d_nadj, d_dLdV, d_dLdc, d_work, s);
    case 2: return launch_adjoint<6>(num_nodes, num_elems, n_states, c, d_nodes, d_elems, d_dofmap, d_psi, d_w, d_nadjptr, d_nadj, d_dLdV, d_dLdc, d_work, s);
    default: return launch_adjoint<10>(num_nodes, num_elems, n_states, c, d_nodes, d_elems, d_dofmap, d_psi, d_w, d_nadjptr, d_nadj, d_dLdV, d_dLdc, d_work, s);
  }
}
