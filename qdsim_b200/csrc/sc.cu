// Self-consistent Poisson-Schrodinger loop, batched over bias points: the
// per-iteration work between the batched eigensolve and the batched Poisson
// solve.  One CTA per bias point for everything that reduces over the mesh,
// so every sum is taken in a fixed order (deterministic).
//
// Layouts: potentials, densities and mixing history are [node][bias]
// (the right-hand-side layout of qd_pcg_solve); the Schrodinger potential of
// the batched eigensolve is [bias][node] (the union mesh, dot b = bias b);
// eigenvectors are the solver's rows x k, rows of bias b at b * R + dof(node).
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include "common.h"

namespace {

constexpr int kSCThreads = 256;
constexpr double kQ = 1.602176634e-19;

__device__ double block_sum(double v, double *s) {
  const int t = threadIdx.x;
  __syncthreads();
  s[t] = v;
  __syncthreads();
  for (int w = kSCThreads / 2; w > 0; w >>= 1) {
    if (t < w) s[t] += s[t + w];
    __syncthreads();
  }
  const double r = s[0];
  __syncthreads();
  return r;
}

// V_out[b][i] = V_static[i] - phi[i][b]  (eV; phi in V)
__global__ void sc_potential_kernel(int nb, int64_t n, const double *__restrict__ Vs,
                                    const double *__restrict__ phi, double *__restrict__ out) {
  const int64_t total = n * nb;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / n, i = e % n;
    out[e] = Vs[i] - phi[i * nb + b];
  }
}

// Densities of self_consistent_solver.pyx:244-286 for bias b = blockIdx.x:
// E_F = E_0 + kT/2, f_s = 1/(1 + exp((E_s - E_F)/kT)) (0 once the exponent
// reaches 50), n = sum_s f_s psi_s^2 rescaled to mean N_D, p = N_A exp(-phi/V_T)
// where phi > 0 else N_A, rho = q (p - n).
__global__ void __launch_bounds__(kSCThreads)
sc_density_kernel(int nb, int64_t n, int k, int64_t rows_per_bias, const int32_t *__restrict__ dof,
                  const double *__restrict__ X, const double *__restrict__ E, double kT,
                  double N_A, double N_D, const double *__restrict__ phi, double *__restrict__ n_out,
                  double *__restrict__ p_out, double *__restrict__ rho_out) {
  __shared__ double s_red[kSCThreads];
  __shared__ double s_f[64];
  const int b = blockIdx.x, t = threadIdx.x;
  if (t < k) {
    const double ef = E[size_t(b) * k] + 0.5 * kT;
    const double a = (E[size_t(b) * k + t] - ef) / kT;
    s_f[t] = a < 50.0 ? 1.0 / (1.0 + exp(a)) : 0.0;
  }
  __syncthreads();
  const double *Xb = X + size_t(b) * rows_per_bias * k;
  double sum = 0.0;
  for (int64_t i = t; i < n; i += kSCThreads) {
    const int r = dof[i];
    double v = 0.0;
    if (r >= 0) {
      const double *x = Xb + size_t(r) * k;
      for (int s = 0; s < k; ++s) v += s_f[s] * x[s] * x[s];
    }
    n_out[i * nb + b] = v;
    sum += v;
  }
  sum = block_sum(sum, s_red);
  const double scale = sum > 0.0 ? N_D / (sum / double(n)) : 1.0;
  for (int64_t i = t; i < n; i += kSCThreads) {
    const double ne = n_out[i * nb + b] * scale;
    const double ph = phi[i * nb + b];
    const double pe = ph > 0.0 ? N_A * exp(-ph / kT) : N_A;   // V_T = kT/q in volts
    n_out[i * nb + b] = ne;
    p_out[i * nb + b] = pe;
    rho_out[i * nb + b] = kQ * (pe - ne);
  }
}

struct MixArgs {
  int nb;
  int64_t n;
  int nhist;                 // entries in the history after this push (Anderson mode)
  int anderson;              // 0: damping only
  const double *old_;        // phi_old
  const double *upd;         // phi_update (the Poisson solution)
  double *hist_upd[3];       // history of updates; slot nhist-1 receives this one
  double *hist_res[3];       // history of residuals upd - old
  double *out;               // phi_new
  double *damping;           // per bias, adapted in place
  double *prev_error;        // per bias
  double *error;             // per bias, output
};

// Mixing of self_consistent.cpp for bias b = blockIdx.x:
//  damping (:1270-1273) phi_new = phi_old + beta (phi_upd - phi_old), beta = 0.3 at start;
//  Anderson (:1291-1419) over the last 3 updates: least squares on residual
//  differences (rank test 1e-10, Tikhonov fallback scaled by the condition
//  number), coefficients clipped to [-2, 2] and their sum to 2, a backtracking
//  line search on || phi_old + s (phi_acc - phi_old) - phi_upd || (:1433-1468),
//  a non-finite / |phi| > 100 guard, then damping of the result;
//  error ||phi_new - phi_old|| / ||phi_new|| and beta *= 0.8 when it grows
//  while beta > 0.1 (:1604, 1644-1647).
__global__ void __launch_bounds__(kSCThreads) sc_mix_kernel(MixArgs a) {
  __shared__ double s_red[kSCThreads];
  __shared__ double s_alpha[2];
  __shared__ double s_step;
  __shared__ int s_mode;   // 0 damping of upd, 1 damping of the line-search point
  const int b = blockIdx.x, t = threadIdx.x, nb = a.nb;
  const int64_t n = a.n;
  const double beta = a.damping[b];
  const bool and_mode = a.anderson && a.nhist >= 1;
  // record this update and its residual in the history
  if (and_mode) {
    double *hu = a.hist_upd[a.nhist - 1], *hr = a.hist_res[a.nhist - 1];
    for (int64_t i = t; i < n; i += kSCThreads) {
      const size_t o = size_t(i) * nb + b;
      hu[o] = a.upd[o];
      hr[o] = a.upd[o] - a.old_[o];
    }
    __syncthreads();
  }
  if (t == 0) s_mode = 0;
  __syncthreads();
  if (and_mode && a.nhist >= 2) {
    const int m = a.nhist - 1;   // columns F_j = r_j - r_m, target -r_m
    const double *rm = a.hist_res[m];
    double d00 = 0, d01 = 0, d11 = 0, c0 = 0, c1 = 0;
    for (int64_t i = t; i < n; i += kSCThreads) {
      const size_t o = size_t(i) * nb + b;
      const double tm = -rm[o];
      const double f0 = a.hist_res[0][o] - rm[o];
      const double f1 = m > 1 ? a.hist_res[1][o] - rm[o] : 0.0;
      d00 += f0 * f0;
      d01 += f0 * f1;
      d11 += f1 * f1;
      c0 += f0 * tm;
      c1 += f1 * tm;
    }
    d00 = block_sum(d00, s_red);
    d01 = block_sum(d01, s_red);
    d11 = block_sum(d11, s_red);
    c0 = block_sum(c0, s_red);
    c1 = block_sum(c1, s_red);
    if (t == 0) {
      double al0 = 0.0, al1 = 0.0;
      bool ok = true;
      if (m == 1) {
        if (d00 > 0.0) {
          al0 = c0 / d00;
        } else {
          ok = false;
        }
      } else {
        // column-pivoted QR from the Gram entries: R00 = |a|, R11 = dist(b, span a)
        const bool swap = d11 > d00;
        const double aa = swap ? d11 : d00, bb = swap ? d00 : d11;
        const double r00 = sqrt(aa);
        const double r11sq = bb - (aa > 0.0 ? d01 * d01 / aa : 0.0);
        const double r11 = sqrt(fmax(r11sq, 0.0));
        if (aa > 0.0 && r11 > 1e-10 * r00) {
          const double det = d00 * d11 - d01 * d01;
          al0 = (d11 * c0 - d01 * c1) / det;
          al1 = (d00 * c1 - d01 * c0) / det;
        } else if (aa > 0.0) {
          // rank-deficient: Tikhonov on the normal equations; singular values of
          // the 2-column F from its Gram matrix
          const double tr = d00 + d11, dt = d00 * d11 - d01 * d01;
          const double disc = sqrt(fmax(0.25 * tr * tr - dt, 0.0));
          const double smax = sqrt(fmax(0.5 * tr + disc, 0.0));
          const double smin = sqrt(fmax(0.5 * tr - disc, 0.0));
          const double cond = smin > 0.0 ? smax / smin : INFINITY;
          const double reg = (cond > 1e8 ? 1e-4 : cond > 1e6 ? 1e-6 : 1e-8) * smax;
          const double e00 = d00 + reg, e11 = d11 + reg;
          const double det = e00 * e11 - d01 * d01;
          al0 = (e11 * c0 - d01 * c1) / det;
          al1 = (e00 * c1 - d01 * c0) / det;
        } else {
          ok = false;
        }
      }
      if (!isfinite(al0) || !isfinite(al1)) ok = false;
      if (ok) {
        al0 = fmax(fmin(al0, 2.0), -2.0);
        al1 = fmax(fmin(al1, 2.0), -2.0);
        const double sum = al0 + al1;
        if (fabs(sum) > 2.0) {
          al0 *= 2.0 / fabs(sum);
          al1 *= 2.0 / fabs(sum);
        }
      }
      s_alpha[0] = al0;
      s_alpha[1] = al1;
      s_mode = ok ? 1 : 0;
    }
    __syncthreads();
    if (s_mode == 1) {
      // phi_acc = upd_m + sum_j alpha_j (upd_j - upd_m); d = phi_acc - old; r = old - upd
      const double al0 = s_alpha[0], al1 = s_alpha[1];
      const double *um = a.hist_upd[m];
      double aa = 0, ad = 0, dd = 0;
      for (int64_t i = t; i < n; i += kSCThreads) {
        const size_t o = size_t(i) * nb + b;
        double acc = um[o] + al0 * (a.hist_upd[0][o] - um[o]);
        if (m > 1) acc += al1 * (a.hist_upd[1][o] - um[o]);
        const double d = acc - a.old_[o], r = a.old_[o] - a.upd[o];
        aa += r * r;
        ad += r * d;
        dd += d * d;
      }
      aa = block_sum(aa, s_red);
      ad = block_sum(ad, s_red);
      dd = block_sum(dd, s_red);
      if (t == 0) {
        const double r0 = sqrt(aa);
        double s = 1.0, chosen = 0.1;
        for (int it = 0; it < 10; ++it) {
          const double tn = sqrt(fmax(aa + 2.0 * s * ad + s * s * dd, 0.0));
          if (tn <= (1.0 - 0.5 * s) * r0) {
            chosen = s;
            break;
          }
          s *= 0.5;
        }
        s_step = chosen;
      }
      __syncthreads();
      // guard: the line-search point must be finite with |phi| <= 100
      int bad = 0;
      for (int64_t i = t; i < n; i += kSCThreads) {
        const size_t o = size_t(i) * nb + b;
        double acc = um[o] + al0 * (a.hist_upd[0][o] - um[o]);
        if (m > 1) acc += al1 * (a.hist_upd[1][o] - um[o]);
        const double v = a.old_[o] + s_step * (acc - a.old_[o]);
        bad |= !(isfinite(v) && fabs(v) <= 100.0);
      }
      bad = __syncthreads_or(bad);
      if (bad) {
        if (t == 0) s_mode = 0;
        __syncthreads();
      }
    }
  }
  // phi_new and the error
  const int mode = s_mode;
  const int m = a.nhist - 1;
  double dn = 0, nn = 0;
  for (int64_t i = t; i < n; i += kSCThreads) {
    const size_t o = size_t(i) * nb + b;
    double target = a.upd[o];
    if (mode == 1) {
      const double *um = a.hist_upd[m];
      double acc = um[o] + s_alpha[0] * (a.hist_upd[0][o] - um[o]);
      if (m > 1) acc += s_alpha[1] * (a.hist_upd[1][o] - um[o]);
      target = a.old_[o] + s_step * (acc - a.old_[o]);
    }
    const double v = a.old_[o] + beta * (target - a.old_[o]);
    a.out[o] = v;
    dn += (v - a.old_[o]) * (v - a.old_[o]);
    nn += v * v;
  }
  dn = block_sum(dn, s_red);
  nn = block_sum(nn, s_red);
  if (t == 0) {
    const double err = nn > 0.0 ? sqrt(dn / nn) : sqrt(dn);
    if (err > a.prev_error[b] && beta > 0.1) a.damping[b] = beta * 0.8;
    a.prev_error[b] = err;
    a.error[b] = err;
  }
}

}  // namespace

extern "C" int qd_sc_potential(int32_t nb, int64_t n_nodes, const double *d_V_static,
                               const double *d_phi, double *d_V_out, void *stream) {
  if (nb <= 0 || n_nodes <= 0 || !d_V_static || !d_phi || !d_V_out) return QD_ERR_INVALID;
  sc_potential_kernel<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(nb, n_nodes, d_V_static,
                                                                         d_phi, d_V_out);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

extern "C" int qd_sc_density(int32_t nb, int64_t n_nodes, int k, int64_t rows_per_bias,
                             const int32_t *d_dof, const double *d_X, const double *d_E,
                             double kT_eV, double N_A, double N_D, const double *d_phi,
                             double *d_n, double *d_p, double *d_rho, void *stream) {
  if (nb <= 0 || n_nodes <= 0 || k < 1 || k > 64 || rows_per_bias <= 0 || !d_dof || !d_X ||
      !d_E || !(kT_eV > 0.0) || !d_phi || !d_n || !d_p || !d_rho)
    return QD_ERR_INVALID;
  sc_density_kernel<<<nb, kSCThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      nb, n_nodes, k, rows_per_bias, d_dof, d_X, d_E, kT_eV, N_A, N_D, d_phi, d_n, d_p, d_rho);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

extern "C" int qd_sc_mix(int32_t nb, int64_t n_nodes, int anderson, int nhist,
                         const double *d_phi_old, const double *d_phi_upd,
                         double *const *h_hist_upd, double *const *h_hist_res, double *d_phi_new,
                         double *d_damping, double *d_prev_error, double *d_error, void *stream) {
  if (nb <= 0 || n_nodes <= 0 || !d_phi_old || !d_phi_upd || !d_phi_new || !d_damping ||
      !d_prev_error || !d_error)
    return QD_ERR_INVALID;
  if (anderson && (nhist < 1 || nhist > 3 || !h_hist_upd || !h_hist_res)) return QD_ERR_INVALID;
  MixArgs a{};
  a.nb = nb;
  a.n = n_nodes;
  a.nhist = anderson ? nhist : 0;
  a.anderson = anderson ? 1 : 0;
  a.old_ = d_phi_old;
  a.upd = d_phi_upd;
  for (int i = 0; i < 3; ++i) {
    a.hist_upd[i] = (anderson && i < nhist) ? h_hist_upd[i] : nullptr;
    a.hist_res[i] = (anderson && i < nhist) ? h_hist_res[i] : nullptr;
    if (anderson && i < nhist && (!a.hist_upd[i] || !a.hist_res[i])) return QD_ERR_INVALID;
  }
  a.out = d_phi_new;
  a.damping = d_damping;
  a.prev_error = d_prev_error;
  a.error = d_error;
  sc_mix_kernel<<<nb, kSCThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
  QD_CHECK_LAUNCH();
  return QD_OK;
}
