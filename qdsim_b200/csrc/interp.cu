// Evaluation of nodal P1/P2/P3 fields of the structured triangular mesh at
// arbitrary points: value, optional gradient and containing element.
//
// Replaces FEInterpolator::interpolate / interpolateWithGradient / findElement
// (backend/src/fe_interpolator.cpp:54-431), which search every element of the
// mesh for each point, and interpolate_field_kernel
// (backend/src/gpu_kernels.cu:352-423), the same linear scan per thread.  On
// the structured mesh the containing cell follows from the coordinates: a
// point well inside the triangle of its own cell is settled by one
// barycentric test; a point near an edge is tested against the triangles of
// the 3 x 3 cells around it in element-index order, and the first whose
// barycentric coordinates are all >= -1e-10 wins.  Both give the element the
// reference's scan over all elements returns (a triangle passing that test
// lies within 1e-10 of a triangle height of the point, so inside that window).
//
// Mesh layout (qdsim_b200/mesh.py, backend/src/mesh.cpp:66-115): lattice of
// NX = p nx + 1 by NY = p ny + 1 nodes, node = iy NX + ix at
// (ix Lx / (p nx), iy Ly / (p ny)); cell (ci, cj) holds elements
// 2 (cj nx + ci) + t with vertices t = 0: (v00, v10, v01), t = 1:
// (v10, v11, v01); local node a sits at the lattice point
// (bc_a . vertices) / p for the integer barycentric multi-index bc_a.
//
// Points outside every element take, as FEInterpolator does, the value of the
// nearest node (first in node order on ties) and a gradient estimated from
// the nodes that share an element with it (inverse-distance weighted
// directional differences, fe_interpolator.cpp:163-270), or zero, as
// interpolate_field_kernel does.
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>
#include "common.h"
#include "interp_shape.cuh"

namespace {

constexpr int kThreads = 128;
constexpr double kInsideEps = 1e-10;
// unique neighbours of a node over the elements that contain it: at most
// 6 triangles x 9 other nodes for P3
constexpr int kMaxLinked = 64;

struct Geo {
  int nx, ny, NX, NY;
  double hx, hy;    // cell size
  double ihx, ihy;  // their reciprocals
  double hxl, hyl;  // lattice spacing
  double margin;    // interior depth that rules out every other triangle
};

// cell-lattice corners (in cell units) of triangle t of cell (ci, cj)
__host__ __device__ __forceinline__ void tri_corners(int ci, int cj, int t, int cx[3], int cy[3]) {
  if (t == 0) {
    cx[0] = ci;     cy[0] = cj;
    cx[1] = ci + 1; cy[1] = cj;
    cx[2] = ci;     cy[2] = cj + 1;
  } else {
    cx[0] = ci + 1; cy[0] = cj;
    cx[1] = ci + 1; cy[1] = cj + 1;
    cx[2] = ci;     cy[2] = cj + 1;
  }
}

// global node index of local node a of triangle (ci, cj, t)
template <int P>
__host__ __device__ __forceinline__ int local_node(const Geo &g, const int cx[3], const int cy[3], int a) {
  int lx = 0, ly = 0;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    lx += Local<P>::b(a, m) * cx[m];
    ly += Local<P>::b(a, m) * cy[m];
  }
  // corners are in cell units, so (bc . P corners) / P = bc . corners
  return ly * g.NX + lx;
}

__host__ __device__ __forceinline__ int clamp_cell(double q, int hi) {
  // fmax/fmin return the other operand for NaN, so NaN lands on cell 0
  return int(fmin(fmax(floor(q), 0.0), double(hi)));
}

// Nearest lattice node to (x, y) by the squared distance, the first in node
// order on ties, or -1 when no distance is below DBL_MAX (non-finite or
// overflowing coordinates), as the reference's scan over all nodes.
__host__ __device__ int nearest_node(const Geo &g, double x, double y) {
  const int jx = clamp_cell(x / g.hxl, g.NX - 1), jy = clamp_cell(y / g.hyl, g.NY - 1);
  double best = DBL_MAX;
  int node = -1;
  for (int iy = max(jy - 1, 0); iy <= min(jy + 1, g.NY - 1); ++iy) {
    const double dy = y - double(iy) * g.hyl;
    for (int ix = max(jx - 1, 0); ix <= min(jx + 1, g.NX - 1); ++ix) {
      const double dx = x - double(ix) * g.hxl;
      const double d = dx * dx + dy * dy;
      if (d < best) {
        best = d;
        node = iy * g.NX + ix;
      }
    }
  }
  return node;
}

// Gradient estimate at a node from the nodes sharing an element with it, in
// the order the reference discovers them (elements ascending, local order),
// each counted once (fe_interpolator.cpp:186-266).
template <int P>
__host__ __device__ __noinline__ void node_gradient(const Geo &g, int node, int nfield, int64_t fstride,
                                           const double *__restrict__ field, int64_t npts,
                                           int64_t i, double *gx, double *gy) {
  const int ix = node % g.NX, iy = node / g.NX;
  const double x0 = double(ix) * g.hxl, y0 = double(iy) * g.hyl;
  int linked[kMaxLinked];
  int nl = 0;
  const int ci0 = max((ix + P - 1) / P - 1, 0), ci1 = min(ix / P, g.nx - 1);
  const int cj0 = max((iy + P - 1) / P - 1, 0), cj1 = min(iy / P, g.ny - 1);
  for (int cj = cj0; cj <= cj1; ++cj)
    for (int ci = ci0; ci <= ci1; ++ci)
      for (int t = 0; t < 2; ++t) {
        int cx[3], cy[3];
        tri_corners(ci, cj, t, cx, cy);
        int self = -1;
        for (int a = 0; a < Local<P>::K && self < 0; ++a)
          if (local_node<P>(g, cx, cy, a) == node) self = a;
        if (self < 0) continue;
        for (int a = 0; a < Local<P>::K; ++a) {
          if (a == self) continue;
          const int q = local_node<P>(g, cx, cy, a);
          bool seen = false;
          for (int s = 0; s < nl; ++s) seen = seen || linked[s] == q;
          if (!seen && nl < kMaxLinked) linked[nl++] = q;
        }
      }
  for (int f = 0; f < nfield; ++f) {
    const double *fv = field + f * fstride;
    const double f0 = fv[node];
    double sx = 0.0, sy = 0.0, wsum = 0.0;
    for (int s = 0; s < nl; ++s) {
      const int q = linked[s];
      const double dx = double(q % g.NX) * g.hxl - x0;
      const double dy = double(q / g.NX) * g.hyl - y0;
      const double dist = sqrt(dx * dx + dy * dy);
      if (dist > 1e-10) {
        const double w = 1.0 / dist;
        const double df = fv[q] - f0;
        sx += w * (df * dx / dist);
        sy += w * (df * dy / dist);
        wsum += w;
      }
    }
    gx[f * npts + i] = wsum > 0.0 ? sx / wsum : 0.0;
    gy[f * npts + i] = wsum > 0.0 ? sy / wsum : 0.0;
  }
}

struct Hit {
  int element, ci, cj, t;
  double l0, l1, l2;
};

// The triangles of the 3 x 3 cells around (ci0, cj0) in element order: the
// first whose barycentric coordinates (signed-area formula) are all >= -1e-10,
// with its cell, t and coordinates; element -1 when there is none.
template <int P>
__host__ __device__ __forceinline__ Hit scan_cells(const Geo &g, double x, double y, int ci0,
                                                int cj0) {
  Hit h{-1, 0, 0, 0, 0.0, 0.0, 0.0};
  for (int cj = max(cj0 - 1, 0); cj <= min(cj0 + 1, g.ny - 1); ++cj)
    for (int ci = max(ci0 - 1, 0); ci <= min(ci0 + 1, g.nx - 1); ++ci)
      for (int t = 0; t < 2; ++t) {
        int cx[3], cy[3];
        double vx[3], vy[3], l[3];
        tri_corners(ci, cj, t, cx, cy);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          vx[m] = double(P * cx[m]) * g.hxl;
          vy[m] = double(P * cy[m]) * g.hyl;
        }
        bary(vx, vy, x, y, l);
        if (l[0] >= -kInsideEps && l[1] >= -kInsideEps && l[2] >= -kInsideEps)
          return Hit{2 * (cj * g.nx + ci) + t, ci, cj, t, l[0], l[1], l[2]};
      }
  return h;
}

// Value (and gradient) of every field and the containing element at point i.
template <int P, bool GRAD>
__host__ __device__ __forceinline__ void interp_point(
    const Geo &g, int nfield, int64_t fstride, const double *__restrict__ field, int64_t npts,
    int64_t i, double x, double y, double *__restrict__ val, double *__restrict__ gx,
    double *__restrict__ gy, int32_t *__restrict__ elem, int outside_zero) {
  constexpr int K = Local<P>::K;
  int found = -1, fcx[3], fcy[3];
  double l[3];
  // Fast path: the triangle of the point's own cell.  A point that lies
  // deeper than g.margin inside it (every barycentric coordinate at least
  // g.margin) is farther from every other triangle than their -1e-10
  // acceptance band reaches, so this is the only element the scan finds.
  // Its barycentric coordinates come from cell-local coordinates measured
  // from the cell's corner, (x - X0) / hx and (y - Y0) / hy, which equal the
  // signed-area formula's up to rounding and carry no cancellation of
  // coordinate-sized terms.
  const int ci0 = clamp_cell(x * g.ihx, g.nx - 1), cj0 = clamp_cell(y * g.ihy, g.ny - 1);
  int t = 0;
  {
    const double u = (x - double(P * ci0) * g.hxl) * g.ihx;
    const double w = (y - double(P * cj0) * g.hyl) * g.ihy;
    t = u + w > 1.0 ? 1 : 0;
    if (t == 0) {
      l[0] = 1.0 - u - w;
      l[1] = u;
      l[2] = w;
    } else {
      l[0] = 1.0 - w;
      l[1] = u + w - 1.0;
      l[2] = 1.0 - u;
    }
    if (l[0] >= g.margin && l[1] >= g.margin && l[2] >= g.margin) {
      found = 2 * (cj0 * g.nx + ci0) + t;
      tri_corners(ci0, cj0, t, fcx, fcy);
    }
  }
  // Otherwise the ordered scan of the 3 x 3 cells around it.
  if (found < 0) {
    const Hit h = scan_cells<P>(g, x, y, ci0, cj0);
    found = h.element;
    if (found >= 0) {
      t = h.t;
      l[0] = h.l0;
      l[1] = h.l1;
      l[2] = h.l2;
      tri_corners(h.ci, h.cj, t, fcx, fcy);
    }
  }
  if (elem) elem[i] = found;
  if (found >= 0) {
    double phi[K], dphi[K][3];
    shape<P>(l, phi, dphi);
    int nodes[K];
#pragma unroll
    for (int a = 0; a < K; ++a) nodes[a] = local_node<P>(g, fcx, fcy, a);
    // gradients of the barycentric coordinates (fe_interpolator.cpp:542-566):
    // every triangle is one of the two right triangles of a cell, so they are
    // +-1/hx and +-1/hy
    double glx[3] = {0, 0, 0}, gly[3] = {0, 0, 0};
    if (GRAD) {
      if (t == 0) {
        glx[0] = -g.ihx; gly[0] = -g.ihy;
        glx[1] = g.ihx;
        gly[2] = g.ihy;
      } else {
        gly[0] = -g.ihy;
        glx[1] = g.ihx; gly[1] = g.ihy;
        glx[2] = -g.ihx;
      }
    }
    for (int f = 0; f < nfield; ++f) {
      const double *fv = field + f * fstride;
      double v = 0.0, sx = 0.0, sy = 0.0;
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const double fa = fv[nodes[a]];
        v += fa * phi[a];
        if (GRAD) {
          const double bx = dphi[a][0] * glx[0] + dphi[a][1] * glx[1] + dphi[a][2] * glx[2];
          const double by = dphi[a][0] * gly[0] + dphi[a][1] * gly[1] + dphi[a][2] * gly[2];
          sx += fa * bx;
          sy += fa * by;
        }
      }
      val[f * npts + i] = v;
      if (GRAD) {
        gx[f * npts + i] = sx;
        gy[f * npts + i] = sy;
      }
    }
    return;
  }
  const int node = outside_zero ? -1 : nearest_node(g, x, y);
  for (int f = 0; f < nfield; ++f) val[f * npts + i] = node >= 0 ? field[f * fstride + node] : 0.0;
  if (GRAD) {
    if (node >= 0) {
      node_gradient<P>(g, node, nfield, fstride, field, npts, i, gx, gy);
    } else {
      for (int f = 0; f < nfield; ++f) gx[f * npts + i] = gy[f * npts + i] = 0.0;
    }
  }
}

template <int P, bool GRAD>
__global__ void __launch_bounds__(kThreads, GRAD ? 4 : 5)
interp_kernel(Geo g, int nfield, int64_t fstride, const double *__restrict__ field, int64_t npts,
              const double *__restrict__ px, const double *__restrict__ py,
              double *__restrict__ val, double *__restrict__ gx, double *__restrict__ gy,
              int32_t *__restrict__ elem, int outside_zero) {
  // the next point's coordinates are loaded before this point's gathers, so
  // the two dependent memory round trips of consecutive points overlap
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double x = 0.0, y = 0.0;
  if (i < npts) {
    x = px[i];
    y = py[i];
  }
  for (; i < npts; i += stride) {
    const int64_t j = i + stride;
    double xn = 0.0, yn = 0.0;
    if (j < npts) {
      xn = px[j];
      yn = py[j];
    }
    interp_point<P, GRAD>(g, nfield, fstride, field, npts, i, x, y, val, gx, gy, elem,
                          outside_zero);
    x = xn;
    y = yn;
  }
}

// Mesh geometry of the launch (arguments already checked).
Geo make_geo(int order, int32_t nx, int32_t ny, double Lx, double Ly) {
  Geo g;
  g.nx = nx;
  g.ny = ny;
  g.NX = order * nx + 1;
  g.NY = order * ny + 1;
  g.hx = Lx / nx;
  g.hy = Ly / ny;
  g.ihx = 1.0 / g.hx;
  g.ihy = 1.0 / g.hy;
  g.hxl = Lx / double(int64_t(order) * nx);
  g.hyl = Ly / double(int64_t(order) * ny);
  // Triangle T' accepts points within 1e-10 of its heights outside it; near
  // a corner of angle a that band reaches 1e-10 h_max / sin(a).  A point at
  // barycentric depth d inside T is at least d h_min from T's boundary, with
  // h_min the height onto the hypotenuse; the band around T' reaches at most
  // 2e-10 h_max / sin(a_min) past it.  d at twice that ratio makes T the only
  // triangle that passes.
  {
    const double hyp = sqrt(g.hx * g.hx + g.hy * g.hy);
    const double hmax = fmax(g.hx, g.hy), hmin = g.hx * g.hy / hyp;
    const double sin_min = fmin(g.hx, g.hy) / hyp;
    g.margin = 4.0 * kInsideEps * hmax / (hmin * sin_min);
  }
  return g;
}

// One wave of resident blocks (grid-stride over the points).
template <int P, bool GRAD>
unsigned resident_blocks() {
  static int blocks = 0;
  if (blocks == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, interp_kernel<P, GRAD>, kThreads,
                                                      0) != cudaSuccess ||
        sms <= 0 || per_sm <= 0)
      return 148u * 4u;
    blocks = sms * per_sm;
  }
  return unsigned(blocks);
}

template <int P>
int launch(const Geo &g, int nfield, int64_t fstride, const double *field, int64_t npts,
           const double *x, const double *y, double *val, double *gx, double *gy, int32_t *elem,
           int outside_zero, cudaStream_t s) {
  const int64_t want = (npts + kThreads - 1) / kThreads;
  if (gx) {
    const unsigned cap = resident_blocks<P, true>();
    const unsigned blocks = unsigned(want < cap ? want : cap);
    interp_kernel<P, true><<<blocks, kThreads, 0, s>>>(g, nfield, fstride, field, npts, x, y, val,
                                                       gx, gy, elem, outside_zero);
  } else {
    const unsigned cap = resident_blocks<P, false>();
    const unsigned blocks = unsigned(want < cap ? want : cap);
    interp_kernel<P, false><<<blocks, kThreads, 0, s>>>(g, nfield, fstride, field, npts, x, y,
                                                        val, nullptr, nullptr, elem, outside_zero);
  }
  QD_CHECK_LAUNCH();
  return QD_OK;
}

}  // namespace

extern "C" int qd_fe_interpolate(int order, int32_t nx, int32_t ny, double Lx, double Ly,
                                 int nfield, int64_t field_stride, const double *d_field,
                                 int64_t npts, const double *d_x, const double *d_y,
                                 double *d_value, double *d_grad_x, double *d_grad_y,
                                 int32_t *d_element, int outside_zero, void *stream) {
  if (order < 1 || order > 3 || nx < 1 || ny < 1 || !(Lx > 0.0) || !(Ly > 0.0) ||
      !(Lx < DBL_MAX) || !(Ly < DBL_MAX) || nfield < 1 || npts < 0 ||
      (outside_zero != 0 && outside_zero != 1) || (d_grad_x == nullptr) != (d_grad_y == nullptr))
    return QD_ERR_INVALID;
  const int64_t NX = int64_t(order) * nx + 1, NY = int64_t(order) * ny + 1;
  // node and element indices are int32
  if (NX * NY > INT32_MAX || 2 * int64_t(nx) * ny > INT32_MAX) return QD_ERR_LIMIT;
  if (field_stride < NX * NY || (npts > 0 && (!d_field || !d_x || !d_y || !d_value)))
    return QD_ERR_INVALID;
  if (npts == 0) return QD_OK;
  const Geo g = make_geo(order, nx, ny, Lx, Ly);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (order) {
    case 1: return launch<1>(g, nfield, field_stride, d_field, npts, d_x, d_y, d_value, d_grad_x, d_grad_y, d_element, outside_zero, s);
    case 2: return launch<2>(g, nfield, field_stride, d_field, npts, d_x, d_y, d_value, d_grad_x, d_grad_y, d_element, outside_zero, s);
    default: return launch<3>(g, nfield, field_stride, d_field, npts, d_x, d_y, d_value, d_grad_x, d_grad_y, d_element, outside_zero, s);
  }
}
