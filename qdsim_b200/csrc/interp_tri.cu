// Evaluation of nodal P1/P2/P3 fields of an unstructured triangular mesh (a
// refined mesh, whose elements no longer follow the lattice) at arbitrary
// points: value, optional gradient and containing element.
//
// Replaces, for such meshes, FEInterpolator::interpolate /
// interpolateWithGradient / findElement (backend/src/fe_interpolator.cpp:
// 54-431), which scan every element for each point.  Point location goes
// through a bucket grid built once on the host: the domain [0, Lx] x [0, Ly]
// is cut into gx x gy cells and each cell lists, in ascending element order,
// the elements whose bounding box (padded by far more than the -1e-10
// acceptance band of the barycentric test) meets it.  Every element the
// reference's scan could accept for a point therefore sits in the bucket of
// the point's cell, and the first element of that bucket that passes the
// test (signed-area formula, every coordinate >= -1e-10) is the first the
// scan over all elements finds.
//
// Points outside every element take the value of the nearest node (squared
// distance, the first in node order on ties; none for non-finite points) and
// the reference's gradient estimate from the nodes sharing an element with it
// (inverse-distance weighted directional differences, each neighbour counted
// once in the order the element scan meets it, fe_interpolator.cpp:163-270),
// or zero with outside_zero (interpolate_field_kernel, gpu_kernels.cu:409-413).
// The nearest node lies within max(hx, hy) of the point's projection onto the
// rectangle (every lattice vertex of the mesh it was refined from is still a
// node), so the search covers the cells within that distance.
#include <cuda_runtime.h>
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include "common.h"
#include "interp_shape.cuh"

namespace {

constexpr int kThreads = 128;
constexpr double kInsideEps = 1e-10;
constexpr int kMaxLinked = 160;   // unique neighbours of a node: <= 16 elements x 9 others

struct TriGrid {
  int gx, gy;          // bucket cells
  double ihx, ihy;     // reciprocal cell size
  int rx, ry;          // cells searched around the point for the nearest node
};

__device__ __forceinline__ int clamp_bucket(double q, int hi) {
  // fmax/fmin return the other operand for NaN, so NaN lands on cell 0
  return int(fmin(fmax(floor(q), 0.0), double(hi)));
}

template <int K>
__device__ __forceinline__ void vertices(const double2 *nodes, const int32_t *elems, int e,
                                         double vx[3], double vy[3]) {
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const double2 p = nodes[elems[size_t(e) * K + m]];
    vx[m] = p.x;
    vy[m] = p.y;
  }
}

template <int P, bool GRAD>
__global__ void __launch_bounds__(kThreads)
interp_tri_kernel(TriGrid g, const double2 *__restrict__ nodes, const int32_t *__restrict__ elems,
                  const int32_t *__restrict__ cell_ptr, const int32_t *__restrict__ cell_elems,
                  const int32_t *__restrict__ nadjptr, const int32_t *__restrict__ nadj,
                  int nfield, int64_t fstride, const double *__restrict__ field, int64_t npts,
                  const double *__restrict__ xs, const double *__restrict__ ys,
                  double *__restrict__ val, double *__restrict__ gxo, double *__restrict__ gyo,
                  int32_t *__restrict__ elem_out, int outside_zero) {
  constexpr int K = Local<P>::K;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < npts;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double x = xs[i], y = ys[i];
    const int ci = clamp_bucket(x * g.ihx, g.gx - 1), cj = clamp_bucket(y * g.ihy, g.gy - 1);
    const int c = cj * g.gx + ci;
    int found = -1;
    double l[3] = {0.0, 0.0, 0.0}, vx[3], vy[3], area = 1.0;
    for (int q = cell_ptr[c]; q < cell_ptr[c + 1]; ++q) {
      const int e = cell_elems[q];
      double tx[3], ty[3], tl[3];
      vertices<K>(nodes, elems, e, tx, ty);
      const double a = bary(tx, ty, x, y, tl);
      if (tl[0] >= -kInsideEps && tl[1] >= -kInsideEps && tl[2] >= -kInsideEps) {
        found = e;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          l[m] = tl[m];
          vx[m] = tx[m];
          vy[m] = ty[m];
        }
        area = a;
        break;                      // ascending order: the first that passes
      }
    }
    if (elem_out) elem_out[i] = found;
    if (found >= 0) {
      double phi[K], dphi[K][3];
      shape<P>(l, phi, dphi);
      int nd[K];
#pragma unroll
      for (int a = 0; a < K; ++a) nd[a] = elems[size_t(found) * K + a];
      // grad lambda_m (fe_interpolator.cpp:552-566)
      const double gl[3][2] = {{0.5 * (vy[1] - vy[2]) / area, 0.5 * (vx[2] - vx[1]) / area},
                               {0.5 * (vy[2] - vy[0]) / area, 0.5 * (vx[0] - vx[2]) / area},
                               {0.5 * (vy[0] - vy[1]) / area, 0.5 * (vx[1] - vx[0]) / area}};
      for (int f = 0; f < nfield; ++f) {
        const double *fv = field + f * fstride;
        double v = 0.0, sx = 0.0, sy = 0.0;
#pragma unroll
        for (int a = 0; a < K; ++a) {
          const double fa = fv[nd[a]];
          v += fa * phi[a];
          if (GRAD) {
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              sx += fa * dphi[a][m] * gl[m][0];
              sy += fa * dphi[a][m] * gl[m][1];
            }
          }
        }
        val[f * npts + i] = v;
        if (GRAD) {
          gxo[f * npts + i] = sx;
          gyo[f * npts + i] = sy;
        }
      }
      continue;
    }
    int node = -1;
    if (!outside_zero) {
      double best = DBL_MAX;
      for (int bj = max(cj - g.ry, 0); bj <= min(cj + g.ry, g.gy - 1); ++bj)
        for (int bi = max(ci - g.rx, 0); bi <= min(ci + g.rx, g.gx - 1); ++bi) {
          const int b = bj * g.gx + bi;
          for (int q = cell_ptr[b]; q < cell_ptr[b + 1]; ++q) {
            const int e = cell_elems[q];
            for (int a = 0; a < K; ++a) {
              const int n = elems[size_t(e) * K + a];
              const double2 p = nodes[n];
              const double dx = x - p.x, dy = y - p.y;
              const double d = dx * dx + dy * dy;
              if (d < best || (d == best && node >= 0 && n < node)) {
                best = d;
                node = n;
              }
            }
          }
        }
    }
    for (int f = 0; f < nfield; ++f) {
      val[f * npts + i] = node >= 0 ? field[f * fstride + node] : 0.0;
      if (GRAD) {
        gxo[f * npts + i] = 0.0;
        gyo[f * npts + i] = 0.0;
      }
    }
    if (GRAD && node >= 0) {
      // neighbours of the node over its elements (ascending), local order
      int linked[kMaxLinked];
      int nl = 0;
      for (int t = nadjptr[node]; t < nadjptr[node + 1]; ++t) {
        const int e = nadj[t] >> 4, self = nadj[t] & 15;
        for (int a = 0; a < K; ++a) {
          if (a == self) continue;
          const int q = elems[size_t(e) * K + a];
          bool seen = false;
          for (int s = 0; s < nl; ++s) seen = seen || linked[s] == q;
          if (!seen && nl < kMaxLinked) linked[nl++] = q;
        }
      }
      const double2 p0 = nodes[node];
      for (int f = 0; f < nfield; ++f) {
        const double *fv = field + f * fstride;
        const double f0 = fv[node];
        double sx = 0.0, sy = 0.0, wsum = 0.0;
        for (int s = 0; s < nl; ++s) {
          const double2 pq = nodes[linked[s]];
          const double dx = pq.x - p0.x, dy = pq.y - p0.y;
          const double dist = sqrt(dx * dx + dy * dy);
          if (dist > 1e-10) {
            const double w = 1.0 / dist;
            const double df = fv[linked[s]] - f0;
            sx += w * (df * dx / dist);
            sy += w * (df * dy / dist);
            wsum += w;
          }
        }
        gxo[f * npts + i] = wsum > 0.0 ? sx / wsum : 0.0;
        gyo[f * npts + i] = wsum > 0.0 ? sy / wsum : 0.0;
      }
    }
  }
}

template <int P>
int launch_tri(const TriGrid &g, const double2 *nodes, const int32_t *elems,
               const int32_t *cell_ptr, const int32_t *cell_elems, const int32_t *nadjptr,
               const int32_t *nadj, int nfield, int64_t fstride, const double *field,
               int64_t npts, const double *x, const double *y, double *val, double *gx,
               double *gy, int32_t *el, int outside_zero, cudaStream_t s) {
  const int blocks = int(std::min<int64_t>((npts + kThreads - 1) / kThreads, 148 * 16));
  if (gx || gy)
    interp_tri_kernel<P, true><<<blocks, kThreads, 0, s>>>(g, nodes, elems, cell_ptr, cell_elems,
                                                           nadjptr, nadj, nfield, fstride, field,
                                                           npts, x, y, val, gx, gy, el,
                                                           outside_zero);
  else
    interp_tri_kernel<P, false><<<blocks, kThreads, 0, s>>>(g, nodes, elems, cell_ptr,
                                                            cell_elems, nadjptr, nadj, nfield,
                                                            fstride, field, npts, x, y, val, gx,
                                                            gy, el, outside_zero);
  QD_CHECK_LAUNCH();
  return QD_OK;
}

}  // namespace

extern "C" int qd_fe_interpolate_tri(int order, int64_t num_nodes, int64_t num_elems,
                                     const double *d_nodes, const int32_t *d_elems,
                                     int32_t grid_nx, int32_t grid_ny, double Lx, double Ly,
                                     const int32_t *d_cell_ptr, const int32_t *d_cell_elems,
                                     const int32_t *d_nadjptr, const int32_t *d_nadj,
                                     int nfield, int64_t field_stride, const double *d_field,
                                     int64_t npts, const double *d_x, const double *d_y,
                                     double *d_value, double *d_grad_x, double *d_grad_y,
                                     int32_t *d_element, int outside_zero, void *stream) {
  if (order < 1 || order > 3 || num_nodes <= 0 || num_elems <= 0 || grid_nx <= 0 ||
      grid_ny <= 0 || !(Lx > 0.0) || !(Ly > 0.0) || nfield < 1 || field_stride < num_nodes ||
      npts < 0)
    return QD_ERR_INVALID;
  if (num_nodes >= (int64_t(1) << 31) || num_elems >= (int64_t(1) << 27) ||
      int64_t(grid_nx) * grid_ny >= (int64_t(1) << 31))
    return QD_ERR_LIMIT;
  if (!d_nodes || !d_elems || !d_cell_ptr || !d_cell_elems || !d_field || !d_value ||
      (npts > 0 && (!d_x || !d_y)) || ((d_grad_x == nullptr) != (d_grad_y == nullptr)) ||
      (d_grad_x && (!d_nadjptr || !d_nadj)))
    return QD_ERR_INVALID;
  if (reinterpret_cast<uintptr_t>(d_nodes) % 16 != 0) return QD_ERR_INVALID;
  if (npts == 0) return QD_OK;
  const double hx = Lx / grid_nx, hy = Ly / grid_ny, h = std::max(hx, hy);
  TriGrid g{grid_nx, grid_ny, 1.0 / hx, 1.0 / hy, int(std::ceil(h / hx)) + 1,
            int(std::ceil(h / hy)) + 1};
  const double2 *nd = reinterpret_cast<const double2 *>(d_nodes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (order) {
    case 1: return launch_tri<1>(g, nd, d_elems, d_cell_ptr, d_cell_elems, d_nadjptr, d_nadj, nfield, field_stride, d_field, npts, d_x, d_y, d_value, d_grad_x, d_grad_y, d_element, outside_zero, s);
    case 2: return launch_tri<2>(g, nd, d_elems, d_cell_ptr, d_cell_elems, d_nadjptr, d_nadj, nfield, field_stride, d_field, npts, d_x, d_y, d_value, d_grad_x, d_grad_y, d_element, outside_zero, s);
    default: return launch_tri<3>(g, nd, d_elems, d_cell_ptr, d_cell_elems, d_nadjptr, d_nadj, nfield, field_stride, d_field, npts, d_x, d_y, d_value, d_grad_x, d_grad_y, d_element, outside_zero, s);
  }
}
